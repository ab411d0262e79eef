"""RunLog -- a JSON-lines run log in place of the reference's FPS console
line (src/main.ts:44-49: "FPS: n, Avg frame time: t ms" once a second).

Each entry is one JSON object per line with the frame rate over the last
interval and the FP64 diagnostics of the simulation's current state
(Simulation.diagnostics): total mass, centre of mass, momentum, angular
momentum, kinetic energy and, when asked for, the direct-sum potential and
total energy with its drift from the first entry.
"""
from __future__ import annotations

import json
import time


class RunLog:
    def __init__(self, sink, sim, potential: bool = True, interval_s: float = 1.0):
        self._own = isinstance(sink, str)
        self._f = open(sink, "a") if self._own else sink
        self.sim = sim
        self.potential = potential
        self.interval_s = interval_s
        self.frames = 0
        self.total_frames = 0
        self._last = time.perf_counter()
        self._t0 = self._last
        self._e0 = None

    def frame(self) -> dict | None:
        """Count one submitted frame (main.ts:43); log once per interval."""
        self.frames += 1
        self.total_frames += 1
        now = time.perf_counter()
        if now - self._last < self.interval_s:
            return None
        return self.log(now=now)

    def log(self, now: float | None = None, **extra) -> dict:
        """Write one entry now (synchronises the simulation's stream)."""
        now = time.perf_counter() if now is None else now
        dt = max(now - self._last, 1e-12)
        entry = {"t_s": now - self._t0, "frames": self.total_frames,
                 "fps": self.frames / dt,
                 "avg_frame_ms": 1e3 * dt / self.frames if self.frames else None,
                 "bodies": self.sim.getNumBodies()}
        d = self.sim.diagnostics(potential=self.potential)
        entry.update(d)
        if self.potential:
            if self._e0 is None:
                self._e0 = d["total_energy"]
            entry["energy_drift"] = ((d["total_energy"] - self._e0) / abs(self._e0)
                                     if self._e0 else 0.0)
        entry.update(extra)
        self._f.write(json.dumps(entry) + "\n")
        self._f.flush()
        self.frames = 0
        self._last = now
        return entry

    def close(self) -> None:
        if self._own and not self._f.closed:
            self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
