"""The reference's Simulation API semantics on the engine (simulation.ts).

frames x substeps steps per submitted frame (simulation.ts:386-425), new
buffers on every body-count or scenario change (:367-369), getBuffers() as
borrowed device views, updateMetadataBuffer() without effect on results,
host state round trips, and argument errors -- all through the C ABI.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(bh, n=3000, **cfg):
    s = bh.Simulation(bh.Config(**cfg))
    s.setNumBodies(n)
    s.setScenario("default", 12)
    return s


def test_frames_times_substeps(bh):
    a = _sim(bh, substeps=3, deltaTime=1e-3)
    b = _sim(bh, substeps=1, deltaTime=1e-3)
    a.step(2)            # 2 frames x 3 substeps
    b.step(6)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


def test_submitted_commands_equal_step(bh):
    a = _sim(bh)
    b = _sim(bh)
    bh.submit([a.getCommands(), a.getCommands()])  # main.ts:38-41
    b.step(2)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


def test_update_metadata_buffer_changes_nothing(bh):
    a = _sim(bh)
    b = _sim(bh)
    a.updateMetadataBuffer()
    a.step(3)
    b.step(3)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


def test_buffers_are_borrowed_views_renewed_on_change(bh):
    s = _sim(bh, n=5000)
    b1 = s.getBuffers()
    assert b1.numBodies == 5000 and b1.pos and b1.mass and b1.stream
    mass, pos, vel = s.download()
    # the handle's device buffers hold the same data as the host copy
    got = s.read_buffer("pos", np.float32, 2 * 5000).reshape(-1, 2)
    assert np.array_equal(got, pos)
    # a new body count reallocates (simulation.ts:367-369): new buffers, new size
    s.setNumBodies(7000)
    b2 = s.getBuffers()
    assert b2.numBodies == 7000 and s.getNumBodies() == 7000
    assert s.download()[1].shape == (7000, 2)
    s.close()


def test_upload_download_round_trip_and_errors(bh):
    s = _sim(bh, n=1000)
    rng = np.random.default_rng(3)
    m = rng.random(1000, dtype=np.float32) + 0.5
    p = rng.standard_normal((1000, 2)).astype(np.float32)
    v = rng.standard_normal((1000, 2)).astype(np.float32)
    s.upload(m, p, v)
    m2, p2, v2 = s.download()
    assert np.array_equal(m, m2) and np.array_equal(p, p2) and np.array_equal(v, v2)
    s.upload(None, p * 2, None)  # NULL skips an array
    m3, p3, v3 = s.download()
    assert np.array_equal(m3, m) and np.array_equal(p3, p * 2) and np.array_equal(v3, v)
    with pytest.raises(ValueError):
        s.upload(m[:10], None, None)  # wrong length
    with pytest.raises(ValueError):
        s.setNumBodies(-1)
    s.close()


def test_zero_bodies_step_and_download(bh):
    s = _sim(bh, n=0)
    s.step(3)
    s.sync()
    m, p, v = s.download()
    assert m.shape == (0,) and p.shape == (0, 2)
    assert s.computeAccelerations().shape == (0, 2)
    s.close()


def _pinned(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).pin_memory()


@pytest.mark.parametrize("integrator,walk", [("symplectic-euler", "group"),
                                             ("symplectic-euler", "exact"),
                                             ("leapfrog-kdk", "group")])
def test_velocity_upload_overlapping_the_tree_stages(bh, integrator, walk):
    """Uploaded velocities cross PCIe on a copy stream while the next step's
    tree stages run; the results must be those of waiting for the upload."""
    cfg = dict(integrator=integrator, walk=walk, softening="plummer", plummerEps=1e-3,
               mortonDomain="bbox", deltaTime=1e-3)
    a = _sim(bh, n=20000, **cfg)
    b = _sim(bh, n=20000, **cfg)
    m, p, v = a.download()
    keep = []  # page-locked host arrays stay alive until the copies are done
    for k in range(3):
        hm, hp, hv = _pinned(m), _pinned(p * (1.0 + 0.01 * k)), _pinned(v * (1.0 + 0.5 * k))
        keep.append((hm, hp, hv))
        a.upload(hm, hp, hv)
        a.step(2)            # no wait between the upload and the step
        b.upload(hm, hp, hv)
        b.sync()             # the upload has landed before the step
        b.step(2)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


def test_velocity_upload_then_other_calls(bh):
    """Every call after an upload sees its velocities: a download, the
    diagnostics, a borrowed-buffer read, and a body-count change."""
    s = _sim(bh, n=4000)
    rng = np.random.default_rng(5)
    v = rng.standard_normal((4000, 2)).astype(np.float32)
    hv = _pinned(v)
    s.upload(None, None, hv)
    assert np.array_equal(s.download()[2], v)
    hv2 = _pinned(2 * v)
    s.upload(None, None, hv2)
    assert np.array_equal(s.read_buffer("vel", np.float32, 8000).reshape(-1, 2), 2 * v)
    m = s.download()[0].astype(np.float64)
    s.upload(None, None, hv)
    d = s.diagnostics(potential=False)
    ke = 0.5 * float(np.sum(m * np.sum(v.astype(np.float64) ** 2, axis=1)))
    assert d["kinetic_energy"] == pytest.approx(ke, rel=1e-9)
    s.upload(None, None, hv2)
    s.setNumBodies(3000)       # reallocates while the copy may be in flight
    s.step(1)
    s.sync()
    assert s.download()[2].shape == (3000, 2)
    s.close()


def test_velocity_upload_overlap_on_an_ensemble(bh):
    """The same overlap on an ensemble handle (its tree stages and walk take
    the per-system paths): bit-equal to waiting for the upload."""
    cfg = bh.Config(walk="group", softening="plummer", plummerEps=1e-3, mortonDomain="bbox",
                    integrator="symplectic-euler", deltaTime=5e-5)
    sizes = [3000, 700, 5000]
    a = bh.Ensemble(sizes, cfg)
    b = bh.Ensemble(sizes, cfg)
    a.setScenarios(None, seed=4)
    b.setScenarios(None, seed=4)
    m, p, v = a.download()
    keep = []
    for k in range(2):
        hm, hp, hv = _pinned(m), _pinned(p), _pinned(v * (1.0 + 0.25 * k))
        keep.append((hm, hp, hv))
        a.upload(hm, hp, hv)
        a.step(2)
        b.upload(hm, hp, hv)
        b.sync()
        b.step(2)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


@pytest.mark.parametrize("n", [1, 2, 300, 12000])
def test_partial_uploads_overlapping_the_step(bh, n):
    """Uploads of some arrays only (each travels on the copy stream into its
    own staging buffer), each followed by a step: bit-equal to waiting for
    the upload, down to one and two bodies."""
    cfg = dict(walk="group", softening="plummer", plummerEps=1e-3, mortonDomain="bbox",
               integrator="symplectic-euler", deltaTime=1e-3)
    a = _sim(bh, n=n, **cfg)
    b = _sim(bh, n=n, **cfg)
    m, p, v = a.download()
    keep = []
    patterns = [(m, p, v), (None, None, 0.5 * v), (1.5 * m, None, None), (None, 1.01 * p, None),
                (m, None, v)]
    for pm, pp, pv in patterns:
        arrs = tuple(None if x is None else _pinned(x) for x in (pm, pp, pv))
        keep.append(arrs)
        a.upload(*arrs)
        a.step(1)
        b.upload(*arrs)
        b.sync()
        b.step(1)
    for x, y in zip(a.download(), b.download()):
        assert np.array_equal(x, y)
    a.close()
    b.close()


@pytest.mark.parametrize("integrator,walk,n", [("symplectic-euler", "group", 20000),
                                               ("symplectic-euler", "exact", 20000),
                                               ("leapfrog-kdk", "group", 20000),
                                               ("symplectic-euler", "group", 1),
                                               ("symplectic-euler", "group", 300)])
def test_pipelined_round_trips_equal_serial(bh, integrator, walk, n):
    """Upload, step and asynchronous download per step with no wait in the
    loop: the staged positions of step k+1 cross PCIe while step k runs and
    the download of step k while step k+1 runs.  Every step's downloaded
    state equals a handle that waits for each copy."""
    cfg = dict(integrator=integrator, walk=walk, softening="plummer", plummerEps=1e-3,
               mortonDomain="bbox", deltaTime=1e-3)
    a = _sim(bh, n=n, **cfg)
    b = _sim(bh, n=n, **cfg)
    m, p, v = a.download()
    inputs = [(_pinned(m * (1.0 + 0.1 * k)), _pinned(p * (1.0 + 0.01 * k)), _pinned(v * (1.0 - 0.2 * k)))
              for k in range(4)]
    outs = [(_pinned(np.zeros_like(p)), _pinned(np.zeros_like(v))) for _ in inputs]
    for (hm, hp, hv), (op, ov) in zip(inputs, outs):
        a.upload(hm, hp, hv)
        a.step(1)
        a.download_into(None, op, ov, wait=False)
    a.sync()
    for (hm, hp, hv), (op, ov) in zip(inputs, outs):
        b.upload(hm, hp, hv)
        b.sync()
        b.step(1)
        _, pb, vb = b.download()
        assert np.array_equal(op.numpy(), pb)
        assert np.array_equal(ov.numpy(), vb)
    a.close()
    b.close()


def test_stepping_with_asynchronous_downloads_into_one_buffer(bh):
    """A trajectory recorded through one pair of host arrays: the downloads
    are written in call order, so after the sync they hold the last step;
    a waiting download after an asynchronous one sees the same state."""
    cfg = dict(walk="group", softening="plummer", plummerEps=1e-3, mortonDomain="bbox",
               integrator="symplectic-euler", deltaTime=1e-3)
    a = _sim(bh, n=5000, **cfg)
    b = _sim(bh, n=5000, **cfg)
    _, p, v = a.download()
    op, ov, om = _pinned(np.zeros_like(p)), _pinned(np.zeros_like(v)), _pinned(np.zeros(5000))
    for _ in range(5):
        a.step(1)
        a.download_into(om, op, ov, wait=False)
    a.sync()
    b.step(5)
    mb, pb, vb = b.download()
    assert np.array_equal(op.numpy(), pb) and np.array_equal(ov.numpy(), vb)
    assert np.array_equal(om.numpy(), mb)
    a.step(1)
    a.download_into(None, op, None, wait=False)
    _, pa, _ = a.download()    # waits for the asynchronous copy first
    b.step(1)
    assert np.array_equal(pa, b.download()[1])
    assert np.array_equal(op.numpy(), pa)
    a.close()
    b.close()


def test_asynchronous_download_then_other_calls(bh):
    """A body-count change, a borrowed-buffer read and closing the handle
    while an asynchronous download may still be copying."""
    s = _sim(bh, n=4000)
    _, p, _ = s.download()
    op = _pinned(np.zeros_like(p))
    s.download_into(None, op, None, wait=False)
    assert np.array_equal(s.read_buffer("pos", np.float32, 8000).reshape(-1, 2), p)
    s.sync()
    assert np.array_equal(op.numpy(), p)
    s.download_into(None, op, None, wait=False)
    s.setNumBodies(3000)       # reallocates while the copy may be in flight
    s.step(1)
    assert s.download()[1].shape == (3000, 2)
    q = _pinned(np.zeros((3000, 2)))
    s.step(1)
    s.download_into(None, q, None, wait=False)
    s.close()                  # waits for the copy before freeing anything
    with pytest.raises(Exception):
        s.download_into(None, q, None, wait=False)  # closed handle
