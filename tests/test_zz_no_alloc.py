"""ptbgpu_density_traces_noalloc: the allocation-free electron count / band
energy for callers that cannot allocate device memory (they own every device
buffer through their own pool, or the device is already full).  It is checked
through the C-ABI against ptbgpu_check_density on two calls in a row, with the
same tolerance as the other FP64 reductions (relative 1e-12).

This file is collected last on purpose: it must pass both in a fresh process
and after every other GPU test has used the library.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _packed_density(s):
    from oracle import ptb_oracle as O
    n = s.ndim
    Pd, _ = O.dense_projector(O.blowsym(n, s.Hvec), O.blowsym(n, s.Svec), s.nel)
    return O.packsym(Pd + 1e-4 * np.eye(n))   # slightly off a projector: traces are not integers


def test_density_traces_noalloc_matches_check_density():
    from ptb_b200 import Context, api, synth
    api.load_library()          # before torch: the library keeps its own cuBLAS / cuSOLVER
    import torch

    systems = [synth.water_cluster(8, seed=5), synth.water_cluster(12, seed=6)]
    with Context(0) as ctx:
        for s in systems:       # two calls in a row (different sizes and contents)
            n = s.ndim
            P = _packed_density(s)
            ref = ctx.check_density(n, P, s.Svec, s.Hvec)
            dP = torch.from_numpy(P).cuda()
            dS = torch.from_numpy(s.Svec).cuda()
            dH = torch.from_numpy(s.Hvec).cuda()
            torch.cuda.synchronize()
            nel, band = api.density_traces_noalloc(0, n, dP.data_ptr(), dS.data_ptr(), dH.data_ptr())
            assert abs(nel - ref.nel) <= 1e-12 * abs(ref.nel)
            assert abs(band - ref.band_energy) <= 1e-12 * abs(ref.band_energy)
            nel2, zero = api.density_traces_noalloc(0, n, dP.data_ptr(), dS.data_ptr(), None)
            assert nel2 == nel and zero == 0.0


def test_density_traces_noalloc_rejects_oversized():
    from ptb_b200 import api
    with pytest.raises(api.PtbGpuError) as ei:
        api.density_traces_noalloc(0, 65537, 1 << 20, 1 << 20)
    assert ei.value.code == api.EINVAL and "65536" in str(ei.value)
