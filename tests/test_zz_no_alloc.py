"""The allocation-free hierarchy build against the engine's own tree stage.

bh_build_hierarchy_static() serves callers that cannot let the library
allocate device memory -- a host that owns the whole GPU heap and hands out
every buffer, or a frame loop that cannot take the device-wide sync of
cudaMalloc/cudaFree.  Here the test plays that caller: it allocates every
input and output buffer itself, calls the entry point twice in a row through
the C ABI, and checks each result against the tree the engine's step built
for the same bodies (index arrays and boxes bit for bit, node mass and COM
within the parity tolerances of test_gpu_parity.py).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATIC_MAX = 262144


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _free_device_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("n,cfg", [
    (120_000, dict(mortonDomain="bbox", softening="plummer", bhTheta=0.5)),
    (120_000, dict(mortonBits=64, softening="plummer", bhTheta=0.5)),
    (STATIC_MAX, dict(mortonDomain="bbox", softening="plummer", bhTheta=0.5)),  # the whole array
    (STATIC_MAX, dict(mortonBits=64, softening="plummer", bhTheta=0.5)),
    (1, dict(mortonDomain="bbox", softening="plummer", bhTheta=0.5)),  # a lone leaf
    (2, dict(mortonDomain="bbox", softening="plummer", bhTheta=0.5)),  # the smallest tree
], ids=["120k-32bit", "120k-64bit", "limit-32bit", "limit-64bit", "n1", "n2"])
def test_static_build_matches_engine_on_two_calls(bh, n, cfg):
    import torch
    lib = bh.load()
    sim = bh.Simulation(bh.Config(**cfg))
    sim.setNumBodies(n)
    sim.setScenario("colliding-disks", 5)
    sim.computeAccelerations()  # the engine's tree stage, on the engine's own buffers
    ref = sim.tree()
    b = sim.getBuffers()
    dev = torch.device("cuda", 0)
    node4 = torch.empty(4 * (2 * n - 1), dtype=torch.float32, device=dev)
    # n == 1 has no internal node: the entry point takes null children / boxes
    children = torch.empty(max(2 * (n - 1), 1), dtype=torch.int32, device=dev)
    parent = torch.empty(2 * n - 1, dtype=torch.int32, device=dev)
    aabb = torch.empty(max(4 * (n - 1), 1), dtype=torch.float32, device=dev)
    bits = sim.config.mortonBits
    for call in range(2):
        for t in (node4, children, parent, aabb):
            t.fill_(-7)  # stale contents must all be overwritten
        free_before = _free_device_bytes()
        rc = lib.bh_build_hierarchy_static(
            ctypes.c_void_p(b.mortonCodes), bits, ctypes.c_void_p(b.bodyIndices),
            ctypes.c_void_p(b.mass), ctypes.c_void_p(b.pos), n, _ptr(node4),
            _ptr(children) if n > 1 else None, _ptr(parent), _ptr(aabb) if n > 1 else None, 1,
            ctypes.c_void_p(b.stream))
        assert rc == 0, lib.bh_global_last_error()
        sim.sync()  # enqueued on the engine's stream
        if call == 1:
            # After the first call (which may load the module holding the
            # static array), a call changes no device allocation.
            assert _free_device_bytes() == free_before, "the entry point allocated device memory"
        got4 = node4.cpu().numpy().reshape(-1, 4)
        got_children = children.cpu().numpy().view(np.uint32)[: 2 * (n - 1)].reshape(-1, 2)
        got_parent = parent.cpu().numpy().view(np.uint32)
        got_aabb = aabb.cpu().numpy()[: 4 * (n - 1)].reshape(-1, 4)
        assert np.array_equal(got_children, ref["children"]), f"call {call}: children differ"
        assert np.array_equal(got_parent, ref["parent"]), f"call {call}: parents differ"
        assert np.array_equal(got_aabb, ref["aabb"]), f"call {call}: boxes differ"
        assert np.array_equal(got4[:, 3], ref["node4"][:, 3]), f"call {call}: lengths differ"
        m_ref = ref["node4"][:, 2]
        assert np.all(np.abs(got4[:, 2] - m_ref) <= 1e-5 * np.abs(m_ref) + 1e-30)
        scale = np.abs(ref["node4"][:, :2]).max(1) + ref["node4"][:, 3]
        assert np.all(np.abs(got4[:, :2] - ref["node4"][:, :2]).max(1) <= 1e-5 * scale + 1e-30)
    sim.close()


def test_static_build_rejects_more_bodies_than_its_scratch(bh):
    lib = bh.load()
    rc = lib.bh_build_hierarchy_static(None, 32, None, None, None, STATIC_MAX + 1, None, None,
                                       None, None, 1, None)
    assert rc == 1  # BH_ERR_INVALID_ARGUMENT
    assert str(STATIC_MAX).encode() in lib.bh_global_last_error()
