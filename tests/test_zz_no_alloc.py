"""The allocation-free kinetic-energy entry point (dg_kinetic_energy_noalloc).

It serves callers that cannot call cudaMalloc -- applications whose device
memory belongs to a framework allocator or a fixed arena -- so the library
keeps its scratch in a static device array.  This test checks it through the
C ABI against the context-based dg_kinetic_energy on the same device state,
twice in a row (the shared scratch array must not carry results from one call
into the next).  The file sorts last so that a first-failure run has already
run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

import dg_b200

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative; FP64 reductions in a different summation order


def test_noalloc_kinetic_energy_matches_context_entry_point():
    import torch

    n, L, p = (6, 5, 4), 2 * np.pi, 3
    mesh = dg_b200.periodic_box(n, (0.0, 0.0, 0.0), (L, L, L))
    case = dg_b200.Case(mesh, p, gas_constant=1.0)
    U0 = case.project_ic("TaylorGreen", [0.1])
    ne = case.ne
    # caller-owned device buffers: per-element det J (uniform box) and the result
    h = np.array([L / n[0], L / n[1], L / n[2]])
    djac = torch.full((ne,), float(np.prod(h / 2.0)), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")

    # the caller's stream, ordered after the context's stream (which wrote the
    # state) by an event, as the header asks
    ctx_stream = torch.cuda.ExternalStream(case.stream_ptr())
    stream = torch.cuda.Stream()
    results = []
    for call in range(2):
        if call == 1:
            case.rk4(case.cfl_time_step(U0, 0.1), 3)  # a different state for the second call
        written = torch.cuda.Event()
        written.record(ctx_stream)
        with torch.cuda.stream(stream):
            out.fill_(-1.0)
        stream.wait_event(written)
        dg_b200.kinetic_energy_noalloc(p, ne, case.device_state_ptr(), djac.data_ptr(), out.data_ptr(),
                                       stream.cuda_stream)
        stream.synchronize()
        ke_ref = case.kinetic_energy()
        ke = float(out.item())
        assert abs(ke - ke_ref) <= TOL * abs(ke_ref), (call, ke, ke_ref)
        results.append(ke)
    assert results[0] != results[1]


def test_noalloc_kinetic_energy_rejects_host_pointers():
    import torch

    ok = torch.zeros(8, dtype=torch.float64, device="cuda")
    host = np.zeros(8)
    with pytest.raises(dg_b200.DGError) as ei:
        dg_b200.kinetic_energy_noalloc(1, 1, host.ctypes.data, ok.data_ptr(), ok.data_ptr())
    assert ei.value.code == 1 and "d_state" in str(ei.value)


def test_noalloc_kinetic_energy_rejects_meshes_beyond_its_scratch():
    with pytest.raises(dg_b200.DGError) as ei:
        dg_b200.kinetic_energy_noalloc(3, 64 * 16384 + 1, 1, 1, 1)
    assert ei.value.code == 1 and "allocation-free limit" in str(ei.value)
