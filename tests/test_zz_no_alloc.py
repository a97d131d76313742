"""vbd_ip_energy_noalloc: the allocation-free incremental-potential entry point.

It serves callers that cannot let a library allocate device memory (code inside a framework that
owns the device memory pool, or a fixed-latency loop where cudaMalloc / cudaFree would synchronise
the device).  Its scratch is a fixed __device__ array, so this test checks it through the C ABI
against the existing vbd_solver_energy(VBD_ENERGY_IP) on two calls in a row (the second call
meets the first call's leftover scratch), and checks the size limit.  It lives in its own file,
collected last, so a run that stops at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

from vbd_tetmesh_b200 import _capi, build_solver, meshgen, precompute_tets
from vbd_tetmesh_b200._capi import VBDError

pytestmark = pytest.mark.gpu

IP_RTOL = 1e-9  # the tolerance of the existing energy tests (FP64 sums, different grouping)


def _dev(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype)).cuda()


def test_noalloc_ip_matches_solver_energy_on_two_calls(gpu_device):
    import torch

    m = meshgen.jittered_block(10, 6, 5, seed=7, per_tet_sigma=0.2)
    s = build_solver(m)
    h = float(np.float32(1.0 / 60.0))
    dm, v0 = precompute_tets(m.rest, m.tets)
    # inputs and the output live in caller-owned device memory (allocated here, by the caller)
    tets = _dev(torch, m.tets, np.int32)
    dmi = _dev(torch, dm.reshape(-1, 9), np.float32)
    vol = _dev(torch, v0, np.float32)
    mu = _dev(torch, m.mu, np.float32)
    lam = _dev(torch, m.lam, np.float32)
    mass = _dev(torch, s.vertex_mass, np.float32)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    results = []
    for call in range(2):
        s.step(1.0 / 60.0, 8, (0.0, -9.8, 0.0), True, 0.9)
        x = _dev(torch, s.get_positions(), np.float32)
        y = _dev(torch, s.get_inertia(), np.float32)
        expected = s.energy(_capi.ENERGY_IP, h)
        _capi.call("vbd_ip_energy_noalloc", m.num_verts, m.num_tets, x.data_ptr(), y.data_ptr(), mass.data_ptr(),
                   tets.data_ptr(), dmi.data_ptr(), vol.data_ptr(), mu.data_ptr(), lam.data_ptr(), h,
                   out.data_ptr(), None)
        got = float(out.cpu()[0])
        assert abs(got - expected) <= IP_RTOL * abs(expected), (call, got, expected)
        results.append(got)
    assert results[0] != results[1]  # two different states, both matched
    s.close()


def test_noalloc_bad_ids_flagged_then_next_call_clean(gpu_device):
    """A tet holding an id outside [0, N) is skipped before any load and reported; the next call,
    on the same scratch (its error flag still set by the failed call), clears the flag and matches
    vbd_solver_energy."""
    import torch

    m = meshgen.jittered_block(6, 4, 4, seed=9, per_tet_sigma=0.2)
    s = build_solver(m)
    h = float(np.float32(1.0 / 60.0))
    s.step(1.0 / 60.0, 8, (0.0, -9.8, 0.0), True, 0.9)
    dm, v0 = precompute_tets(m.rest, m.tets)
    bad = m.tets.copy()
    bad[3, 2] = m.num_verts       # one past the end
    bad[7, 0] = -5                # negative
    args = [_dev(torch, a, np.float32) for a in (s.get_positions(), s.get_inertia(), s.vertex_mass)]
    rest = [_dev(torch, dm.reshape(-1, 9), np.float32), _dev(torch, v0, np.float32), _dev(torch, m.mu, np.float32),
            _dev(torch, m.lam, np.float32)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    tets_bad = _dev(torch, bad, np.int32)
    with pytest.raises(VBDError) as e:
        _capi.call("vbd_ip_energy_noalloc", m.num_verts, m.num_tets, *[a.data_ptr() for a in args],
                   tets_bad.data_ptr(), *[a.data_ptr() for a in rest], h, out.data_ptr(), None)
    assert e.value.code == 1 and f"outside [0, {m.num_verts})" in e.value.message
    tets = _dev(torch, m.tets, np.int32)
    _capi.call("vbd_ip_energy_noalloc", m.num_verts, m.num_tets, *[a.data_ptr() for a in args], tets.data_ptr(),
               *[a.data_ptr() for a in rest], h, out.data_ptr(), None)
    expected = s.energy(_capi.ENERGY_IP, h)
    assert abs(float(out.cpu()[0]) - expected) <= IP_RTOL * abs(expected)
    s.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_device):
    out = C.c_double(0.0)
    with pytest.raises(VBDError) as e:
        _capi.call("vbd_ip_energy_noalloc", 16_000_000, 1_000_000, None, None, None, None, None, None, None, None,
                   0.01, C.addressof(out), None)
    assert e.value.code == 1 and "exceeds the no-alloc maximum" in e.value.message
