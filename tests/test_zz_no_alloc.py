"""The allocation-free statistics entry point, cel_stats_noalloc.

It exists for callers that must not allocate device memory when they ask for the statistics (a
frame loop that cannot afford the device-wide synchronisation of an allocation, an application
whose own allocator has reserved the device's memory).  The tests hand it a state and a bottom that
live in device memory and check two calls in a row against the statistics the engine's own
resetTimestep path returns for the same state: a small plain-form state, and a state of the largest
domain the fixed scratch accepts (1024 x 1024 interior cells, 65,536 4x4 blocks) from both the plain
and the compensated form.  A domain larger than the scratch is refused.  This file is collected last
so that a run stopping at the first failure has run every other test before it.
"""
from __future__ import annotations

import ctypes as C

import pytest

from celeris_b200 import abi, cases

pytestmark = pytest.mark.gpu

# resetTimestep reports the CFL rate after its time-step choice; the other totals come from the same
# per-block partials and the same FP64 reduction order, so they agree to the last bit.
KEYS = ["mass", "x_momentum", "y_momentum", "kinetic_energy", "potential_energy", "total_energy",
        "max_speed", "max_depth", "max_froude", "mass_full"]


def _noalloc(lib, d_state, d_bottom, params, stream_ptr):
    out = abi.Stats()
    st = lib.cel_stats_noalloc(C.c_void_p(d_state), C.c_void_p(d_bottom), C.byref(params), C.c_void_p(stream_ptr),
                               C.byref(out))
    return st, out.as_dict()


def test_stats_noalloc_matches_reset_timestep(celeris):
    import torch
    lib = celeris.lib()
    p, z, bnx, bny = cases.small_case(96, 64, "mixed", correction_steps=1)
    eng = celeris.Engine(p, z, "plain")
    eng.physical_steps(40)
    ref = eng.reset_timestep()          # statistics of the current state, through the engine
    state = torch.from_numpy(eng.state()).cuda()
    bottom = torch.from_numpy(eng.bottom()).cuda()
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    for _ in range(2):                  # two calls in a row share the same scratch
        st, got = _noalloc(lib, state.data_ptr(), bottom.data_ptr(), p, stream.cuda_stream)
        assert st == 0, lib.cel_last_error().decode()
        for k in KEYS:
            assert got[k] == pytest.approx(ref[k], rel=1e-12, abs=1e-30), k
        assert got["cfl_rate"] > 0
        assert got["health"] == 0


def test_stats_noalloc_rejects_oversized_domain(celeris):
    import torch
    lib = celeris.lib()
    p = abi.default_params()
    p.nx, p.ny = 2048, 1024             # 131,072 4x4 blocks > the 65,536 the scratch holds
    dummy = torch.zeros(4, device="cuda")
    st, _ = _noalloc(lib, dummy.data_ptr(), dummy.data_ptr(), p, 0)
    assert st == 1                      # CEL_ERR_ARG
    assert b"scratch" in lib.cel_last_error()


@pytest.mark.parametrize("form, rel", [("plain", 1e-12), ("mixed", 1e-5)])
def test_stats_noalloc_at_the_largest_accepted_domain(celeris, form, rel):
    """1024 x 1024 interior cells: exactly the 65,536 blocks the scratch holds.  The compensated
    form's own totals come from its stencil's reduction (FP32 Kahan sums per thread) and its volume
    includes the low words, so they agree with the float state's totals to rounding only."""
    import torch
    lib = celeris.lib()
    p, z, bnx, bny = cases.config3(1024, 1024)
    eng = celeris.Engine(p, z, form)
    eng.physical_steps(3)
    ref = eng.reset_timestep()
    state = torch.from_numpy(eng.state()).cuda()
    bottom = torch.from_numpy(eng.bottom()).cuda()
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    for _ in range(2):
        st, got = _noalloc(lib, state.data_ptr(), bottom.data_ptr(), p, stream.cuda_stream)
        assert st == 0, lib.cel_last_error().decode()
        for k in KEYS:
            if k in ("x_momentum", "y_momentum"):   # sums of signed terms: judged on their scale
                assert abs(got[k] - ref[k]) <= rel * max(abs(ref["mass"]), 1e-30), k
            else:
                assert got[k] == pytest.approx(ref[k], rel=rel, abs=1e-30), k
        assert got["health"] == 0
