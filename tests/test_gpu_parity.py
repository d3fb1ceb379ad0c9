"""GPU parity: every entry point of libptbgpu.so against the CPU oracle.

Tolerances: FP64 paths agree with the oracle to rounding of different
(but equally FP64) LAPACK/BLAS implementations; the mixed-precision
trace-correcting path meets max|dP| <= 1e-6, |dE| <= 1e-6 Eh and the electron
count to 1e-8 against the FP64 dense projector.
"""
import numpy as np
import pytest

from oracle import ptb_oracle as O
from ptb_b200 import PREC_FP64, PREC_MIXED, Options, PtbGpuError, PurificationSettings, synth
from ptb_b200 import api

pytestmark = pytest.mark.gpu

TOL_P = 1e-6        # max |dP|
TOL_E = 1e-6        # |d tr(PH)| in Eh
TOL_NEL = 1e-8      # |tr(PS) - nel|


def emulate_bf16x3_square(X):
    """X @ X with the kernel's operand rounding: hi = bf16(x), lo = bf16(x - hi), (hh + hl + lh)."""
    def bf16(a):
        a = np.asarray(a, np.float32)
        b = a.view(np.uint32).astype(np.uint64)
        b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
        return b.astype(np.uint32).view(np.float32).astype(np.float64)
    x32 = np.asarray(X, np.float32)
    h = bf16(x32)
    l = bf16(x32.astype(np.float64) - h)
    return h @ h + h @ l + l @ h


@pytest.mark.parametrize("n", [64, 256, 300, 700])
def test_symsq_bf16x3_matches_emulation(ctx, n):
    rng = np.random.default_rng(n)
    A = rng.uniform(-1, 1, (n, n))
    X = 0.5 * (A + A.T)
    C = ctx.symsq_bf16x3(X).astype(np.float64)
    ref = emulate_bf16x3_square(X)
    # FP32 accumulation of n split products: |fl(sum) - sum| <= n u sum|terms| (u = 2^-24)
    bound = n * 2.0 ** -24 * (np.abs(X) @ np.abs(X)) + 1e-30
    assert np.all(np.abs(C - ref) <= bound)
    # and against the exact product (operand split error ~2^-16 relative)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(C - X @ X)) <= 1e-4 * scale


@pytest.mark.parametrize("planes", [2, 3])
@pytest.mark.parametrize("kblock", [32, 64])
def test_symsq_both_k_blocks(ctx, planes, kblock):
    """Both K-block variants of the kernel (64B / 128B swizzle) give the same product."""
    n = 520
    rng = np.random.default_rng(7)
    A = rng.uniform(-1, 1, (n, n))
    X = 0.5 * (A + A.T)
    C = ctx.symsq_split(X, planes, kblock).astype(np.float64)
    ref = ctx.symsq_split(X, planes, 64 if kblock == 32 else 32).astype(np.float64)
    bound = 2 * n * 2.0 ** -24 * (np.abs(X) @ np.abs(X)) + 1e-30
    assert np.all(np.abs(C - ref) <= bound)
    assert np.max(np.abs(C - X @ X)) <= 1e-4 * np.max(np.abs(X @ X))


@pytest.mark.parametrize("kblock", [1032, 1064])
@pytest.mark.parametrize("n", [256, 520, 1100])
def test_symsq_cta_pair_kernel(ctx, kblock, n):
    """The cta_group::2 kernel (256 x 256 tiles over two SMs) gives the
    one-CTA product to FP32 accumulation accuracy, on sizes that pad."""
    rng = np.random.default_rng(n + kblock)
    A = rng.uniform(-1, 1, (n, n))
    X = 0.5 * (A + A.T)
    C = ctx.symsq_split(X, 2, kblock).astype(np.float64)
    ref = ctx.symsq_split(X, 2, 64).astype(np.float64)
    bound = 2 * n * 2.0 ** -24 * (np.abs(X) @ np.abs(X)) + 1e-30
    assert np.all(np.abs(C - ref) <= bound)
    assert np.max(np.abs(C - X @ X)) <= 1e-4 * np.max(np.abs(X @ X))


@pytest.mark.parametrize("n", [200, 512, 640])
def test_symsq_bf16x6_three_plane_split(ctx, n):
    rng = np.random.default_rng(n + 1)
    A = rng.uniform(-1, 1, (n, n))
    X = 0.5 * (A + A.T)
    C = ctx.symsq_bf16x6(X).astype(np.float64)

    def bf16(a):
        a = np.asarray(a, np.float32)
        b = a.view(np.uint32).astype(np.uint64)
        b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
        return b.astype(np.uint32).view(np.float32)
    x32 = X.astype(np.float32)
    h = bf16(x32)
    r = (x32 - h).astype(np.float32)
    m = bf16(r)
    lo = bf16((r - m).astype(np.float32))
    h, m, lo = (v.astype(np.float64) for v in (h, m, lo))
    emu = h @ h + h @ m + m @ h + h @ lo + lo @ h + m @ m
    # the six products of the three planes, up to FP32 accumulation
    bound = n * 2.0 ** -24 * (np.abs(X) @ np.abs(X)) + 1e-30
    assert np.all(np.abs(C - emu) <= bound)
    # off the diagonal the three-plane product is closer to the exact FP32-operand
    # product than the two-plane one (the tensor-core accumulation error is of the
    # same order as the two-plane split error, so the gain is a factor ~1.3-3)
    exact = x32.astype(np.float64) @ x32.astype(np.float64)
    off = ~np.eye(n, dtype=bool)
    C3 = ctx.symsq_bf16x3(X).astype(np.float64)
    assert np.median(np.abs(C - exact)[off]) < 0.9 * np.median(np.abs(C3 - exact)[off])


def test_filter_packed_bit_exact(ctx, water8):
    s = water8
    out = ctx.filter_matrix_sym(s.Hvec, s.ndim, 1e-3)
    assert np.array_equal(out, O.filter_matrix_sym(s.Hvec, 1e-3))


def test_check_density_matches_oracle(ctx, water8):
    s = water8
    n = s.ndim
    H, S = O.blowsym(n, s.Hvec), O.blowsym(n, s.Svec)
    Pd, _ = O.dense_projector(H, S, s.nel)
    P = Pd + 1e-4 * np.eye(n)
    st = ctx.check_density(n, O.packsym(P), s.Svec, s.Hvec)
    Ps = O.blowsym(n, O.packsym(P))
    ref_q, ref_f = O.idempotency_deviation(Ps, S)
    assert abs(st.nel - O.get_nel(Ps, S)) < 1e-10
    assert abs(st.band_energy - O.band_structure(Ps, H)) < 1e-10
    assert abs(st.idempotency_ref - ref_q) < 1e-9 * max(1.0, ref_q)
    assert abs(st.idempotency_frob - ref_f) < 1e-9 * max(1.0, ref_f)


@pytest.mark.parametrize("columns", [1, 2, 3, 4])
def test_sm_stupid_simple_matches_oracle(ctx, water8, columns):
    s = water8
    n = s.ndim
    H = O.filter_matrix_sym(s.Hvec, 1e-4)
    S = O.filter_matrix_sym(s.Svec, 1e-4)
    part = None
    if columns == 4:
        part = (np.arange(s.nat) // 6 % 3 + 1).astype(np.int64)   # three clusters
    ref = O.sm_stupid_simple(n, s.nel, H, S, s.nat, s.xyz, s.aoat, columns, 2, part)
    P, st = ctx.sm_stupid_simple(n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, columns, 2, part,
                                 Options(filter=1e-4))
    assert st.nsm == ref.nsm
    assert st.sum_dims == sum(ref.dims)
    assert st.mu == ref.mu
    assert st.mu_iterations == len(ref.mu_trace)
    assert abs(st.nel - ref.nel) < 1e-9
    assert np.max(np.abs(P - ref.Pvec)) < 1e-9


def test_sm_full_matrix_equals_dense_solve2(ctx, water32):
    s = water32
    n = s.ndim
    P, st = ctx.sm_stupid_simple(n, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 3, 2, None, Options(filter=1e-4))
    P2, e, focc, st2 = ctx.solve2(1, n, s.nel, 0, s.Hvec, s.Svec, Options(filter=1e-4))
    assert st.nsm == 1
    assert np.max(np.abs(P - P2)) < 1e-10
    ref, e_ref, f_ref, _ = O.solve2(1, n, s.nel, 0, 300.0, O.filter_matrix_sym(s.Hvec, 1e-4),
                                    O.filter_matrix_sym(s.Svec, 1e-4))
    assert np.max(np.abs(P2 - ref)) < 1e-10
    assert np.max(np.abs(e - e_ref)) < 1e-10
    assert np.max(np.abs(focc - f_ref)) < 1e-10


def test_sm_errors(ctx, water8):
    s = water8
    with pytest.raises(PtbGpuError) as ei:
        ctx.sm_stupid_simple(s.ndim, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 2, 1)
    assert ei.value.code == api.ENOTIMPL
    bad_part = np.zeros(s.nat, dtype=np.int64)   # cluster ids are 1-based
    with pytest.raises(PtbGpuError) as ei:
        ctx.sm_stupid_simple(s.ndim, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 4, 2, bad_part)
    assert ei.value.code == api.EINVAL
    bad = s.Svec.copy()
    bad[0] = -1.0   # S_11 < 0: not positive definite
    with pytest.raises(PtbGpuError) as ei:
        ctx.sm_stupid_simple(s.ndim, s.nel, s.Hvec, bad, s.nat, s.xyz, s.aoat, 3, 2)
    assert ei.value.code == api.ENOTSPD


@pytest.mark.parametrize("ptype,metric,iterative", [(1, 1, False), (1, 2, False), (2, 2, False), (3, 2, False),
                                                    (4, 2, False), (4, 1, False), (3, 1, False), (2, 2, True),
                                                    (3, 1, True)])
def test_purification_matches_oracle(ctx, ptype, metric, iterative):
    s = synth.water_cluster(4, seed=2)
    n = s.ndim
    pur = PurificationSettings(type=ptype, metric_type=metric, metric_iterative=iterative, nel=s.nel, cycles=100,
                               metric_cycles=200)
    ref_pur = O.PurificationSettings(type=ptype, metric_type=metric, metric_iterative=iterative, nel=s.nel,
                                     cycles=100, metric_cycles=200)
    ref, mu, steps = O.purification(ref_pur, n, s.Hvec, s.Svec)
    P, st = ctx.purification(pur, n, s.Hvec, s.Svec)
    assert st.mu_iterations == steps
    assert abs(st.mu - mu) < 1e-9
    assert np.max(np.abs(P - ref)) < 1e-7


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_tc_purify_against_dense(ctx, water32, precision):
    s = water32
    n = s.ndim
    H = O.filter_matrix_sym(s.Hvec, 1e-5)
    S = O.filter_matrix_sym(s.Svec, 1e-5)
    Hf, Sf = O.blowsym(n, H), O.blowsym(n, S)
    Pd, _ = O.dense_projector(Hf, Sf, s.nel)
    P, st = ctx.tc_purify(n, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=precision))
    Pf = O.blowsym(n, P)
    assert np.max(np.abs(P - O.packsym(Pd))) <= TOL_P
    assert abs(O.band_structure(Pf, Hf) - O.band_structure(Pd, Hf)) <= TOL_E
    assert abs(O.get_nel(Pf, Sf) - s.nel) <= TOL_NEL
    assert st.iterations > 10


def test_tc_purify_mixed_larger(ctx):
    s = synth.water_cluster(96, seed=4)
    n = s.ndim
    Hf = O.blowsym(n, O.filter_matrix_sym(s.Hvec, 1e-5))
    Sf = O.blowsym(n, O.filter_matrix_sym(s.Svec, 1e-5))
    Pd, _ = O.dense_projector(Hf, Sf, s.nel)
    P, st = ctx.tc_purify(n, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=PREC_MIXED))
    Pf = O.blowsym(n, P)
    assert np.max(np.abs(Pf - Pd)) <= TOL_P
    assert abs(O.band_structure(Pf, Hf) - O.band_structure(Pd, Hf)) <= TOL_E
    assert abs(O.get_nel(Pf, Sf) - s.nel) <= TOL_NEL


def test_tc_purify_device_pointers_match_host_path(water32):
    """The device-resident entry point on a fresh context (its first scratch
    buffers are claimed without the host path's packed staging buffers)."""
    import torch
    from ptb_b200 import Context
    s = water32
    n = s.ndim
    dH = torch.from_numpy(s.Hvec).cuda()
    dS = torch.from_numpy(s.Svec).cuda()
    dP = torch.empty(n * (n + 1) // 2, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    with Context(0) as fresh:
        for prec in (PREC_FP64, PREC_MIXED):
            st = fresh.tc_purify_device(n, s.nel, dH.data_ptr(), dS.data_ptr(), dP.data_ptr(),
                                        Options(filter=1e-5, precision=prec))
            Pdev = dP.cpu().numpy()
            Phost, _ = fresh.tc_purify(n, s.nel, s.Hvec, s.Svec, Options(filter=1e-5, precision=prec))
            assert np.max(np.abs(Pdev - Phost)) < 1e-12
            assert st.ms_h2d == 0.0 or st.ms_h2d < 1.0


def test_tc_purify_errors(ctx, water8):
    s = water8
    with pytest.raises(PtbGpuError) as ei:
        ctx.tc_purify(s.ndim, s.nel + 1, s.Hvec, s.Svec)
    assert ei.value.code == api.EINVAL
    bad = s.Hvec.copy()
    bad[5] = np.nan
    with pytest.raises(PtbGpuError) as ei:
        ctx.tc_purify(s.ndim, s.nel, bad, s.Svec, Options(precision=PREC_FP64))
    assert ei.value.code == api.ENAN
    with pytest.raises(PtbGpuError) as ei:
        ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(precision=PREC_MIXED, max_iter=3))
    assert ei.value.code == api.EITER
    # the context stays usable after errors
    P, st = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(precision=PREC_MIXED))
    assert abs(st.ms_total) > 0


def test_bounded_wait_reports_timeout_and_context_survives(ctx, water8):
    """A device wait on a flag that nothing sets gives up after its limit and
    comes back as ETIMEOUT (the path every tensor-core pipeline wait takes);
    the same context then runs a purification normally."""
    with pytest.raises(PtbGpuError) as ei:
        ctx.selftest_bounded_wait(20000)
    assert ei.value.code == api.ETIMEOUT
    assert "site 90" in str(ei.value)
    s = water8
    P, st = ctx.tc_purify(s.ndim, s.nel, s.Hvec, s.Svec, Options(precision=PREC_FP64))
    assert st.iterations > 5
    with pytest.raises(PtbGpuError) as ei:
        ctx.selftest_bounded_wait(0)
    assert ei.value.code == api.EINVAL


def test_progress_output_parses_like_the_reference(ctx, water8, capfd):
    """At print level 1 the submatrix step and solve2 print the lines the
    reference's result collector reads (collect_and_plot_results.py): the
    'number of submatrices=' line and the closing 'Submatrix' and
    '* sygvd solver' timer lines in the reference's timer layout."""
    s = water8
    P, st = ctx.sm_stupid_simple(s.ndim, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, 2, 2, None,
                                 Options(filter=1e-4, print_level=1))
    ctx.solve2(1, s.ndim, s.nel, 0, s.Hvec, s.Svec, Options(filter=1e-4, print_level=1))
    out = capfd.readouterr().out.splitlines()
    nsm = [int(l.split()[3]) for l in out if l.startswith(" number of submatrices=")]
    tsm = [float(l.split()[1]) for l in out if l.startswith("Submatrix ")]
    tsy = [float(l.split()[3]) for l in out if l.startswith("* sygvd solver")]
    tso = [float(l.split()[2]) for l in out if l.startswith("Total solve2")]
    assert nsm == [st.nsm]
    assert len(tsm) == 1 and tsm[0] > 0.0
    assert len(tsy) == 1 and len(tso) == 1 and 0.0 < tsy[0] <= tso[0]
