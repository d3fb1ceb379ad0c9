"""ptbgpu_density_traces_noalloc: the allocation-free electron count / band
energy for callers that cannot allocate device memory (they own every device
buffer through their own pool, or the device is already full).

It is checked through the C-ABI against ptbgpu_check_density (the library's
context path) and against the oracle's get_nel / band_structure
(source/metrics.f90:182-277) on two calls in a row, with the same tolerance as
the other FP64 reductions (relative 1e-12); on a caller's stream; for device
memory left unchanged by a call; and at its 65536 size limit.

This file is collected last on purpose: it must pass both in a fresh process
and after every other GPU test has used the library.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12


def _packed_density(s):
    from oracle import ptb_oracle as O
    n = s.ndim
    Pd, _ = O.dense_projector(O.blowsym(n, s.Hvec), O.blowsym(n, s.Svec), s.nel)
    return O.packsym(Pd + 1e-4 * np.eye(n))   # slightly off a projector: traces are not integers


def test_density_traces_noalloc_matches_check_density_and_oracle():
    from oracle import ptb_oracle as O
    from ptb_b200 import Context, api, synth
    api.load_library()          # before torch: the library keeps its own cuBLAS / cuSOLVER
    import torch

    systems = [synth.water_cluster(8, seed=5), synth.water_cluster(12, seed=6)]
    with Context(0) as ctx:
        for s in systems:       # two calls in a row (different sizes and contents)
            n = s.ndim
            P = _packed_density(s)
            ref = ctx.check_density(n, P, s.Svec, s.Hvec)
            Pf, Sf, Hf = O.blowsym(n, P), O.blowsym(n, s.Svec), O.blowsym(n, s.Hvec)
            nel_o, band_o = O.get_nel(Pf, Sf), O.band_structure(Pf, Hf)
            dP = torch.from_numpy(P).cuda()
            dS = torch.from_numpy(s.Svec).cuda()
            dH = torch.from_numpy(s.Hvec).cuda()
            torch.cuda.synchronize()
            nel, band = api.density_traces_noalloc(0, n, dP.data_ptr(), dS.data_ptr(), dH.data_ptr())
            assert abs(nel - ref.nel) <= REL * abs(ref.nel)
            assert abs(band - ref.band_energy) <= REL * abs(ref.band_energy)
            assert abs(nel - nel_o) <= REL * abs(nel_o)
            assert abs(band - band_o) <= REL * abs(band_o)
            nel2, zero = api.density_traces_noalloc(0, n, dP.data_ptr(), dS.data_ptr(), None)
            assert nel2 == nel and zero == 0.0
            assert torch.cuda.current_device() == 0


def test_density_traces_noalloc_on_a_stream_allocates_nothing():
    """On a caller's (non-default) stream the result is the same, and a call
    leaves the device's free memory unchanged (the first call on the device,
    which may load the code, has been made before the measurement)."""
    from ptb_b200 import api, synth
    api.load_library()
    import torch

    s = synth.water_cluster(10, seed=7)
    n = s.ndim
    P = _packed_density(s)
    dP = torch.from_numpy(P).cuda()
    dS = torch.from_numpy(s.Svec).cuda()
    dH = torch.from_numpy(s.Hvec).cuda()
    torch.cuda.synchronize()
    first = api.density_traces_noalloc(0, n, dP.data_ptr(), dS.data_ptr(), dH.data_ptr())
    st = torch.cuda.Stream()
    free0, _ = torch.cuda.mem_get_info(0)
    on_stream = api.density_traces_noalloc(0, n, dP.data_ptr(), dS.data_ptr(), dH.data_ptr(),
                                           stream=st.cuda_stream)
    again = api.density_traces_noalloc(0, n, dP.data_ptr(), dS.data_ptr(), dH.data_ptr(),
                                       stream=st.cuda_stream)
    free1, _ = torch.cuda.mem_get_info(0)
    assert on_stream == first and again == first
    assert free1 == free0


def test_density_traces_noalloc_at_the_size_limit():
    """ndim = 65536 (the scratch array's limit), P = S = H packed with seeded
    values; the expected traces are the weighted sums over both triangles."""
    from ptb_b200 import api
    api.load_library()
    import torch

    n = 65536
    npk = n * (n + 1) // 2
    g = torch.Generator(device="cuda").manual_seed(11)
    dP = torch.rand(npk, dtype=torch.float64, device="cuda", generator=g) - 0.5
    dS = torch.rand(npk, dtype=torch.float64, device="cuda", generator=g) - 0.5
    diag = torch.arange(n, device="cuda", dtype=torch.int64)
    diag = diag * (diag + 3) // 2          # packed offset of (j, j): j(j+1)/2 + j
    prod = dP * dS
    expect = float(2.0 * prod.sum() - prod[diag].sum())
    del prod
    torch.cuda.synchronize()
    for _ in range(2):
        nel, _ = api.density_traces_noalloc(0, n, dP.data_ptr(), dS.data_ptr(), None)
        assert abs(nel - expect) <= 1e-9 * float(torch.sqrt(torch.tensor(float(npk))))
    del dP, dS
    torch.cuda.empty_cache()


def test_density_traces_noalloc_rejects_oversized():
    from ptb_b200 import api
    with pytest.raises(api.PtbGpuError) as ei:
        api.density_traces_noalloc(0, 65537, 1 << 20, 1 << 20)
    assert ei.value.code == api.EINVAL and "65536" in str(ei.value)
