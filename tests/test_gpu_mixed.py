"""GPU: the split-TF32 tensor-core GEMM and the mixed-precision refined
solver against FP64 references.

Tolerances: the GEMM on TF32-representable operands with FP32 accumulation
agrees with an FP64 product to 1e-5 relative (K = 384); the mixed solver's
currents agree with the cuSOLVER FP64 path to 1e-9 relative and its
relative residual on the scaled system is <= 1e-10 (the refinement target)."""

import math
import os

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def _tf32(x):
    b = np.asarray(x, dtype=np.float32).view(np.uint32) & np.uint32(0xFFFFE000)
    return b.view(np.float32)


@pytest.mark.parametrize("slots", ["4", "1"])
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("m2,n", [(256, 128), (300, 200), (1000, 517), (4096, 1500)])
def test_gemm_tf32_sub(mode, m2, n, slots, gpu_ctx, monkeypatch):
    """Every kernel mode, with the persistent kernel's C tile in four slots of
    32 columns (default) or one slot of 128 (SIEB200_GEMM_C_SLOTS=1)."""
    import torch
    import sieb200
    from sieb200 import _lib
    if mode < 2 and slots == "1":
        pytest.skip("the slot count applies to the persistent kernel only")
    monkeypatch.setenv("SIEB200_GEMM_C_SLOTS", slots)
    rng = np.random.default_rng(m2 + n)
    K = 384
    A = _tf32(rng.standard_normal((m2, K)))
    B = _tf32(rng.standard_normal((n, K)))
    ldc = m2 + 8
    C = rng.standard_normal((n, ldc)).astype(np.float32)  # column-major storage: C[col, row]
    dA, dB, dC = (torch.from_numpy(x.copy()).cuda() for x in (A, B, C))
    torch.cuda.synchronize()
    _lib.check(_lib.lib().sieb200_gemm_tf32_sub(gpu_ctx.handle, m2, n, K, dA.data_ptr(), dB.data_ptr(),
                                                 dC.data_ptr(), ldc, mode))
    out = dC.cpu().numpy()
    ref = C.astype(np.float64).copy()
    ref[:, :m2] -= (A.astype(np.float64) @ B.astype(np.float64).T).T
    assert rel_err(out[:, :m2], ref[:, :m2]) < 1e-5
    assert np.array_equal(out[:, m2:], C[:, m2:])  # padding rows untouched


@pytest.mark.parametrize("slots", ["4", "1"])
@pytest.mark.parametrize("mode", [4, 5])
@pytest.mark.parametrize("m2,n,K", [(256, 128, 256), (300, 200, 256), (1000, 517, 512), (4096, 1500, 256)])
def test_gemm_tf32_sub_split_operands(mode, m2, n, K, slots, gpu_ctx, monkeypatch):
    """Split operands [hi | lo] along k (modes 4 and 5): C -= A_hi B_hi^T +
    A_hi B_lo^T + A_lo B_hi^T with TF32 hi parts and FP32 remainders, against
    the FP64 product of the unsplit FP32 operands. Tolerance 1e-5 (the
    dropped lo*lo term and FP32 accumulation; a plain TF32 product of these
    operands is off by ~1e-3)."""
    import torch
    from sieb200 import _lib
    monkeypatch.setenv("SIEB200_GEMM_C_SLOTS", slots)
    rng = np.random.default_rng(m2 + n + K)
    KR = K // 2
    A = rng.standard_normal((m2, KR)).astype(np.float32)
    B = rng.standard_normal((n, KR)).astype(np.float32)
    Ah, Bh = _tf32(A), _tf32(B)
    Ap = np.concatenate([Ah, A - Ah], axis=1)
    Bp = np.concatenate([Bh, B - Bh], axis=1)
    ldc = m2 + 8
    C = rng.standard_normal((n, ldc)).astype(np.float32)
    dA, dB, dC = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (Ap, Bp, C))
    torch.cuda.synchronize()
    _lib.check(_lib.lib().sieb200_gemm_tf32_sub(gpu_ctx.handle, m2, n, K, dA.data_ptr(), dB.data_ptr(),
                                                 dC.data_ptr(), ldc, mode))
    out = dC.cpu().numpy()
    ref = C.astype(np.float64).copy()
    ref[:, :m2] -= (A.astype(np.float64) @ B.astype(np.float64).T).T
    assert rel_err(out[:, :m2], ref[:, :m2]) < 1e-5
    assert np.array_equal(out[:, m2:], C[:, m2:])  # padding rows untouched


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("m2,n,shift", [(256, 128, 64), (384, 448, 64), (1000, 517, 64), (300, 200, 137),
                                        (4096, 1600, 64)])
def test_gemm_tf32_sub_shifted(mode, m2, n, shift, gpu_ctx):
    """The first 128 rows of C take columns [shift, n) only (the trailing
    update that leaves the next diagonal block alone); the other rows take
    all n. (384, 448, 64) and (4096, 1600, 64) leave the first row tile's
    last column tile wholly past n (448 - 64 and 1600 - 64 fit in one tile
    fewer), which the kernels skip. Every mode, plain (0-3, K = 384) and
    split (4-5, K = 256) operands; tolerance 1e-5 as above, the untouched
    block bit-exact."""
    import torch
    from sieb200 import _lib
    rng = np.random.default_rng(m2 + n + shift + mode)
    if mode >= 4:
        K = 256
        A32 = rng.standard_normal((m2, K // 2)).astype(np.float32)
        B32 = rng.standard_normal((n, K // 2)).astype(np.float32)
        Ah, Bh = _tf32(A32), _tf32(B32)
        A = np.concatenate([Ah, A32 - Ah], axis=1)
        B = np.concatenate([Bh, B32 - Bh], axis=1)
        prod = A32.astype(np.float64) @ B32.astype(np.float64).T
    else:
        K = 384
        A = _tf32(rng.standard_normal((m2, K)))
        B = _tf32(rng.standard_normal((n, K)))
        prod = A.astype(np.float64) @ B.astype(np.float64).T
    ldc = m2 + 8
    C = rng.standard_normal((n, ldc)).astype(np.float32)
    dA, dB, dC = (torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (A, B, C))
    torch.cuda.synchronize()
    _lib.check(_lib.lib().sieb200_gemm_tf32_sub_shifted(gpu_ctx.handle, m2, n, K, dA.data_ptr(), dB.data_ptr(),
                                                         dC.data_ptr(), ldc, mode, shift))
    out = dC.cpu().numpy()
    ref = C.astype(np.float64).copy()
    ref[:, :m2] -= prod.T
    r1 = min(128, m2)
    ref[:shift, :r1] = C[:shift, :r1]
    assert np.array_equal(out[:shift, :r1], C[:shift, :r1])  # the skipped block
    assert rel_err(out[:, :m2], ref[:, :m2]) < 1e-5
    assert np.array_equal(out[:, m2:], C[:, m2:])  # padding rows untouched


def test_gemm_shift_out_of_range_refused(gpu_ctx):
    import torch
    import sieb200
    from sieb200 import _lib
    d = torch.zeros(256 * 128, device="cuda")
    with pytest.raises(sieb200.SiebError):
        _lib.check(_lib.lib().sieb200_gemm_tf32_sub_shifted(gpu_ctx.handle, 256, 128, 256, d.data_ptr(),
                                                             d.data_ptr(), d.data_ptr(), 256, 3, 128))


def _pmchwt(level=2, solver="lu_cusolver", rule=5):
    import sieb200
    m = sieb200.icosphere(0.5, level)
    o = sieb200.DielectricOptions(frequency_hz=C0, quadrature_rule=rule,
                                  interior=sieb200.IsotropicMedium(4.0, 1.0), solver=solver)
    return m, o


@pytest.mark.parametrize("trailing", ["tc", "tc_pair", "tc_three_product", "tc_load_store", "tc_reduce",
                                      "tc_overlap", "tc_no_lcol", "tc_lcol_gemm", "tc_simt_gemm", "simt"])
def test_mixed_solver_matches_fp64(trailing, gpu_ctx, monkeypatch):
    import sieb200
    if trailing == "tc_no_lcol":  # the next panels update the next block column
        monkeypatch.setenv("SIEB200_GEMM_LCOL", "0")
    if trailing == "tc_lcol_gemm":  # the GEMM does, its first block row shifted
        monkeypatch.setenv("SIEB200_GEMM_LCOL", "1")
    if trailing == "tc_simt_gemm":  # GEMM mode 0 on the same packs and shapes
        monkeypatch.setenv("SIEB200_GEMM_MODE", "0")
    if trailing == "simt":
        monkeypatch.setenv("SIEB200_TRAILING_SIMT", "1")
    if trailing == "tc_pair":
        monkeypatch.setenv("SIEB200_PAIR_UPDATE", "1")
    if trailing == "tc_three_product":
        monkeypatch.setenv("SIEB200_GEMM_HILO", "0")
    if trailing == "tc_overlap":
        monkeypatch.setenv("SIEB200_OVERLAP_MIN", "64")
    if trailing in ("tc_load_store", "tc_reduce"):
        monkeypatch.setenv("SIEB200_GEMM_MODE", "2" if trailing == "tc_load_store" else "3")
    m, o = _pmchwt(2)
    ref = sieb200.solve_dielectric_dense(m, o, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    o.solver = "mixed_ir"
    r = sieb200.solve_dielectric_dense(m, o, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    assert r.metrics["relative_residual"] <= 1e-10
    assert np.linalg.norm(r.currents - ref.currents) / np.linalg.norm(ref.currents) < 1e-9
    assert 1 <= r.metrics["refinement_iterations"] <= 20


def test_mixed_gstc_batch_and_pec(gpu_ctx):
    import sieb200
    m = sieb200.icosphere(1.0, 2)
    rng = np.random.default_rng(2)
    t = rng.standard_normal((m.num_faces, 32)) + 1j * rng.standard_normal((m.num_faces, 32))
    t *= 0.3
    o = sieb200.GstcSieOptions(frequency_hz=C0, quadrature_rule=5)
    cases = [sieb200.GstcExcitationCase(exterior=sieb200.PlaneWaveExcitation()),
             sieb200.GstcExcitationCase(exterior=sieb200.PlaneWaveExcitation(
                 electric_amplitude=(0, 1, 0), propagation_direction=(1, 0, 0)))]
    ref = sieb200.solve_gstc_dense_batch(m, t, o, cases, ctx=gpu_ctx)
    o.solver = "mixed_ir"
    got = sieb200.solve_gstc_dense_batch(m, t, o, cases, ctx=gpu_ctx)
    for a, b in zip(got, ref):
        assert a.metrics["relative_residual"] <= 1e-10
        assert np.linalg.norm(a.currents - b.currents) / np.linalg.norm(b.currents) < 1e-9
    pm = sieb200.icosphere(1.0, 2)
    po = sieb200.PecOptions(frequency_hz=C0, quadrature_rule=5)
    pref = sieb200.solve_pec_dense(pm, po, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    po.solver = "mixed_ir"
    pgot = sieb200.solve_pec_dense(pm, po, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    assert pgot.metrics["relative_residual"] <= 1e-10
    assert np.linalg.norm(pgot.currents - pref.currents) / np.linalg.norm(pref.currents) < 1e-9


def test_dense_solver_object_on_device_memory(gpu_ctx):
    import torch
    import sieb200
    m, o = _pmchwt(2)
    N = 2 * m.num_edges
    Z = torch.empty((N, N), dtype=torch.complex128, device="cuda")
    sieb200.assemble_matrix_device(m, o, Z.data_ptr(), ctx=gpu_ctx)
    b = torch.from_numpy(sieb200.assemble_rhs(m, o, [sieb200.PlaneWaveExcitation()], ctx=gpu_ctx)[:, 0].copy()).cuda()
    Zh = Z.cpu().numpy().T  # storage is column-major
    x_ref = np.linalg.solve(Zh, b.cpu().numpy())
    s = sieb200.DenseLuSolver(N, "mixed_ir", ctx=gpu_ctx)
    s.factorize(Z.data_ptr())
    x = b.clone()
    torch.cuda.synchronize()
    it = s.solve(x.data_ptr(), tolerance=1e-12, max_iterations=60)
    gpu_ctx.synchronize()
    xs = x.cpu().numpy()
    assert np.linalg.norm(xs - x_ref) / np.linalg.norm(x_ref) < 1e-10
    assert np.linalg.norm(Zh @ xs - b.cpu().numpy()) / np.linalg.norm(b.cpu().numpy()) < 1e-12
    assert it >= 1
    s.close()


@pytest.mark.parametrize("schedule", ["pair_split", "single_split", "pair_three", "single_three",
                                      "single_split_overlap", "single_split_trsv64", "pair_then_single",
                                      "single_split_no_lcol", "single_split_lcol_gemm",
                                      "single_split_lcol_side", "single_split_diag_rec",
                                      "single_split_diag_compact", "single_split_trsv_stream"])
@pytest.mark.parametrize("n", [5, 64, 100, 129, 190, 256, 300, 1000, 2100])
def test_mixed_ragged_sizes_one_step(n, schedule, gpu_ctx, monkeypatch):
    """Sizes that leave partial sub-blocks, a last row block with one
    sub-block, and fewer rows than one block, under both trailing-update
    schedules (pair / single step), both pack layouts (split [hi | lo] /
    three-product), the next block column's update in single steps from the
    GEMM (default), the column kernel before or beside it or the panels,
    diagonal blocks by the one-pass 64 x 64 kernel (unrolled or compact)
    or the 32 x 32 recursion,
    with overlapped steps (panels beside the GEMM), with
    64-row triangular-solve CTAs, and switching from the pair to the single
    schedule part way. One preconditioned step must already reach 1e-5 (the
    factors are single precision), and the full refinement 1e-12: a wrong
    triangular solve fails the first bound."""
    import torch
    import sieb200
    monkeypatch.setenv("SIEB200_PAIR_UPDATE", "1" if schedule.startswith("pair_") and schedule != "pair_then_single"
                       else "0")
    # pair steps while the paired update is at least 128 columns wide, single steps after
    monkeypatch.setenv("SIEB200_PAIR_MIN", "128" if schedule == "pair_then_single" else "0")
    monkeypatch.setenv("SIEB200_GEMM_HILO", "0" if "_three" in schedule else "1")
    # overlapped steps: every trailing update at least 64 columns wide skips
    # the next block row, whose update the next panels take on the side stream
    monkeypatch.setenv("SIEB200_OVERLAP_MIN", "64" if schedule.endswith("overlap") else "0")
    monkeypatch.setenv("SIEB200_OVERLAP_SMS", "16")
    # triangular solves with 64-row CTAs (one sub-block each) or 128-row ones
    monkeypatch.setenv("SIEB200_TRSV_ROWS", "64" if schedule.endswith("trsv64") else "128")
    # 128-row triangular solves with the newest coupling folded into
    # precomputed products (default) or streamed as tiles
    monkeypatch.setenv("SIEB200_TRSV_FOLD", "0" if schedule.endswith("trsv_stream") else "1")
    # who updates the next block column below its diagonal block in a single
    # step: the next panels (0), the GEMM (1, default), col_update_kernel on
    # the third stream (2) or before the GEMM (3)
    monkeypatch.setenv("SIEB200_GEMM_LCOL", "0" if schedule.endswith("no_lcol")
                       else "1" if schedule.endswith("lcol_gemm")
                       else "2" if schedule.endswith("lcol_side") else "1")
    # diagonal blocks by the one-pass 64 x 64 kernel, fully unrolled
    # (default) or in one code path, or by the 2 x 2 recursion over 32 x 32
    # warp factorizations
    monkeypatch.setenv("SIEB200_DIAG_REC", "1" if schedule.endswith("diag_rec") else "0")
    monkeypatch.setenv("SIEB200_DIAG_COMPACT", "1" if schedule.endswith("diag_compact") else "0")
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3.0 * math.sqrt(n) * np.eye(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Z = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()  # column-major storage
    s = sieb200.DenseLuSolver(n, "mixed_ir", ctx=gpu_ctx)
    s.factorize(Z.data_ptr())
    x = torch.from_numpy(b.copy()).cuda()
    torch.cuda.synchronize()
    it = s.solve(x.data_ptr(), tolerance=1e-5, max_iterations=1)
    gpu_ctx.synchronize()
    xs = x.cpu().numpy()
    assert it == 1
    assert np.linalg.norm(A @ xs - b) / np.linalg.norm(b) <= 1e-5
    x = torch.from_numpy(b.copy()).cuda()
    torch.cuda.synchronize()
    s.solve(x.data_ptr(), tolerance=1e-12, max_iterations=20)
    gpu_ctx.synchronize()
    xs = x.cpu().numpy()
    assert np.linalg.norm(A @ xs - b) / np.linalg.norm(b) <= 1e-12
    s.close()


_CHAIN_VARIANTS = {
    # (SIEB200_GEMM_LCOL, SIEB200_DIAG_SPLIT, SIEB200_DIAG_PANELS, SIEB200_DIAG_COMPACT)
    "reference": ("3", "1", "0", "1"),
    "panel_updates_column": ("0", "1", "0", "1"),
    "column_update_third_stream": ("2", "1", "0", "1"),
    "fused_diag_update": ("3", "0", "0", "1"),
    "diag_barrier_per_panel": ("3", "1", "1", "1"),
    "diag_unrolled": ("3", "1", "0", "0"),
    "all_previous": ("0", "0", "0", "0"),
}


@pytest.mark.parametrize("n", [64, 130, 1000, 2100])
def test_mixed_split_panels_bit_identical(n, gpu_ctx, monkeypatch):
    """Split panels (SIEB200_PANEL_HEAD_MAX): the next block's rows and
    columns of L21 / U12 in a head launch on the lookahead stream, the rest
    on the context stream. Every 32-row block of the panels runs the same
    code whichever launch it is in, so the factors, and with them the
    one-step solution, are the same bit for bit as with one panels launch:
    for every step split, for the narrower steps only (the switch inside
    the factorization), and with the head's larger shared-memory request."""
    import torch
    import sieb200
    rng = np.random.default_rng(400 + n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3.0 * math.sqrt(n) * np.eye(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Z = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()
    monkeypatch.setenv("SIEB200_PAIR_MIN", "0")
    monkeypatch.setenv("SIEB200_GEMM_LCOL", "1")
    variants = {"one_launch": ("0", "0"), "all_split": ("1000000", "0"),
                "narrow_split": (str(max(1, n // 2)), "0"), "all_split_big_smem": ("1000000", str(200 * 1024))}
    out = {}
    for name, (head_max, smem) in variants.items():
        monkeypatch.setenv("SIEB200_PANEL_HEAD_MAX", head_max)
        if smem == "0":
            monkeypatch.delenv("SIEB200_PANEL_HEAD_SMEM", raising=False)
        else:
            monkeypatch.setenv("SIEB200_PANEL_HEAD_SMEM", smem)
        s = sieb200.DenseLuSolver(n, "mixed_ir", ctx=gpu_ctx)
        xs = []
        for _ in range(3):  # eager, captured, replayed
            s.factorize(Z.data_ptr())
            x = torch.from_numpy(b.copy()).cuda()
            torch.cuda.synchronize()
            s.solve(x.data_ptr(), tolerance=1e-5, max_iterations=1)
            gpu_ctx.synchronize()
            xs.append(x.cpu().numpy())
        s.close()
        for x in xs[1:]:
            assert np.array_equal(x, xs[0]), name
        out[name] = xs[0]
    assert np.linalg.norm(A @ out["one_launch"] - b) / np.linalg.norm(b) <= 1e-5
    for name, xs in out.items():
        assert np.array_equal(xs, out["one_launch"]), name


@pytest.mark.parametrize("n", [64, 200, 1000, 2100])
def test_mixed_chain_variants_bit_identical(n, gpu_ctx, monkeypatch):
    """The chain variants only move work between kernels and streams: the
    next block column's update by col_update_kernel (before the GEMM or on
    a third stream beside it) or by the panels, the diagonal block's update
    by diag_update_kernel or inside the LU kernel, and the elimination with
    a barrier per step (unrolled or in one code path) or per panel all run
    the same FP32 operations in the same order, so the factors, and with
    them the one-step solution, are the same bit for bit."""
    import torch
    import sieb200
    rng = np.random.default_rng(300 + n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3.0 * math.sqrt(n) * np.eye(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Z = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()
    monkeypatch.setenv("SIEB200_PAIR_MIN", "0")
    monkeypatch.setenv("SIEB200_DIAG_REC", "0")  # the one-pass 64 x 64 kernel in every variant
    out = {}
    for name, (lcol, split, panels, compact) in _CHAIN_VARIANTS.items():
        monkeypatch.setenv("SIEB200_GEMM_LCOL", lcol)
        monkeypatch.setenv("SIEB200_DIAG_SPLIT", split)
        monkeypatch.setenv("SIEB200_DIAG_PANELS", panels)
        monkeypatch.setenv("SIEB200_DIAG_COMPACT", compact)
        s = sieb200.DenseLuSolver(n, "mixed_ir", ctx=gpu_ctx)
        s.factorize(Z.data_ptr())
        x = torch.from_numpy(b.copy()).cuda()
        torch.cuda.synchronize()
        s.solve(x.data_ptr(), tolerance=1e-5, max_iterations=1)
        gpu_ctx.synchronize()
        out[name] = x.cpu().numpy()
        s.close()
    assert np.linalg.norm(A @ out["reference"] - b) / np.linalg.norm(b) <= 1e-5
    for name, xs in out.items():
        assert np.array_equal(xs, out["reference"]), name


@pytest.mark.parametrize("rows", ["128", "128_stream", "64"])
@pytest.mark.parametrize("n", [5, 129, 300, 1000])
def test_mixed_adjoint_solve(n, rows, gpu_ctx, monkeypatch):
    """Conjugate-transpose solve A^H x = b with the mixed factors: one
    preconditioned step reaches 1e-5, the refinement 1e-12, as for A x = b
    (triangular solves with 128-row CTAs, the newest coupling folded into
    precomputed products or streamed, and with 64-row CTAs)."""
    import torch
    import sieb200
    monkeypatch.setenv("SIEB200_TRSV_ROWS", rows.split("_")[0])
    monkeypatch.setenv("SIEB200_TRSV_FOLD", "0" if rows.endswith("stream") else "1")
    rng = np.random.default_rng(100 + n)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3.0 * math.sqrt(n) * np.eye(n)
    A[0, n - 1] += 5.0  # make A far from Hermitian
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    AH = A.conj().T
    Z = torch.from_numpy(A.T.copy()).cuda()  # column-major storage of A
    s = sieb200.DenseLuSolver(n, "mixed_ir", ctx=gpu_ctx)
    s.factorize(Z.data_ptr())
    for tol, maxit, bound in [(1e-5, 1, 1e-5), (1e-12, 20, 1e-12)]:
        x = torch.from_numpy(b.copy()).cuda()
        torch.cuda.synchronize()
        s.solve(x.data_ptr(), tolerance=tol, max_iterations=maxit, adjoint=True)
        gpu_ctx.synchronize()
        xs = x.cpu().numpy()
        assert np.linalg.norm(AH @ xs - b) / np.linalg.norm(b) <= bound
    # a forward solve after the adjoint one still uses the untransposed factors
    x = torch.from_numpy(b.copy()).cuda()
    torch.cuda.synchronize()
    s.solve(x.data_ptr(), tolerance=1e-12, max_iterations=20)
    gpu_ctx.synchronize()
    assert np.linalg.norm(A @ x.cpu().numpy() - b) / np.linalg.norm(b) <= 1e-12
    s.close()


def test_mixed_adjoint_matches_cusolver_on_pmchwt(gpu_ctx):
    import torch
    import sieb200
    m, o = _pmchwt(2)
    N = 2 * m.num_edges
    Z = torch.empty((N, N), dtype=torch.complex128, device="cuda")
    sieb200.assemble_matrix_device(m, o, Z.data_ptr(), ctx=gpu_ctx)
    rng = np.random.default_rng(7)
    g = torch.from_numpy(rng.standard_normal(N) + 1j * rng.standard_normal(N)).cuda()
    Zc = Z.clone()
    ref = sieb200.DenseLuSolver(N, "lu_cusolver", ctx=gpu_ctx)
    ref.factorize(Zc.data_ptr())
    lam_ref = g.clone()
    torch.cuda.synchronize()
    ref.solve(lam_ref.data_ptr(), adjoint=True)
    mix = sieb200.DenseLuSolver(N, "mixed_ir", ctx=gpu_ctx)
    mix.factorize(Z.data_ptr())
    lam = g.clone()
    torch.cuda.synchronize()
    mix.solve(lam.data_ptr(), tolerance=1e-12, max_iterations=40, adjoint=True)
    gpu_ctx.synchronize()
    a, r = lam.cpu().numpy(), lam_ref.cpu().numpy()
    assert np.linalg.norm(a - r) / np.linalg.norm(r) < 1e-9
    ref.close()
    mix.close()


@pytest.mark.parametrize("pair", ["0", "1"])
def test_profile_timeline_orders_the_block_steps(pair, gpu_ctx, monkeypatch):
    """The profiler's timeline: one span per hot launch with start <= end,
    every chain kernel inside the factorization span, one diagonal-block
    kernel per block, one panels launch per block step and one tensor-core
    trailing update per step but the last two (single-step schedule) or per
    odd step among those (pair schedule)."""
    import torch
    import sieb200
    monkeypatch.setenv("SIEB200_PAIR_UPDATE", pair)
    n = 1000
    rng = np.random.default_rng(7)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3.0 * math.sqrt(n) * np.eye(n)
    Z = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()
    s = sieb200.DenseLuSolver(n, "mixed_ir", ctx=gpu_ctx)
    gpu_ctx.profile(True, timeline=True)
    s.factorize(Z.data_ptr())
    gpu_ctx.synchronize()
    spans = gpu_ctx.profile_timeline()
    gpu_ctx.profile(False)
    s.close()
    assert spans and all(t0 <= t1 for _, t0, t1 in spans)
    fact = [sp for sp in spans if sp[0] == 6]
    assert len(fact) == 1
    f0, f1 = fact[0][1], fact[0][2]
    inner = [sp for sp in spans if sp[0] in (0, 3, 4)]
    assert all(f0 - 1e-3 <= t0 and t1 <= f1 + 1e-3 for _, t0, t1 in inner)
    nbl = -(-n // 64)
    assert sum(1 for sp in spans if sp[0] == 3) == nbl
    assert sum(1 for sp in spans if sp[0] == 4) == nbl - 1
    # the last two steps have no columns right of the next block
    expect = (nbl - 2) // 2 if pair == "1" else nbl - 2
    assert sum(1 for sp in spans if sp[0] == 0) == expect
    diag = sorted(t0 for k, t0, _ in spans if k == 3)
    assert diag == [t0 for k, t0, _ in spans if k == 3]  # recorded in step order


def test_factorization_graph_replay_matches_eager(gpu_ctx, monkeypatch):
    """The factorization is captured as a CUDA graph on its second call with
    the same operand and replayed after that: the factors (seen through a
    one-step preconditioned solve) are bit-identical to the eager run's. With
    the profiler on it runs eagerly again and every span is recorded."""
    import torch
    import sieb200
    n = 700
    rng = np.random.default_rng(11)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3.0 * math.sqrt(n) * np.eye(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Z = torch.from_numpy(np.asfortranarray(A).T.copy()).cuda()

    def one_step(solver):  # one preconditioned step applies the factors once
        x = torch.from_numpy(b.copy()).cuda()
        torch.cuda.synchronize()
        assert solver.solve(x.data_ptr(), tolerance=1e-5, max_iterations=1) == 1
        gpu_ctx.synchronize()
        return x.cpu().numpy()

    monkeypatch.setenv("SIEB200_NO_GRAPHS", "1")
    s0 = sieb200.DenseLuSolver(n, "mixed_ir", ctx=gpu_ctx)
    s0.factorize(Z.data_ptr())
    ref = one_step(s0)
    s0.close()
    monkeypatch.delenv("SIEB200_NO_GRAPHS")
    s1 = sieb200.DenseLuSolver(n, "mixed_ir", ctx=gpu_ctx)
    launches = []
    for _ in range(4):  # eager, capture + launch, replay, replay
        l0 = sieb200.lib().sieb200_launch_count()
        s1.factorize(Z.data_ptr())
        launches.append(sieb200.lib().sieb200_launch_count() - l0)
        assert np.array_equal(one_step(s1), ref)
    assert launches[0] == launches[1] == launches[2] == launches[3] > 0
    # alternating between two copies of the operand keeps one graph for each
    Z2 = Z.clone()
    for i in range(6):
        s1.factorize((Z2 if i % 2 == 0 else Z).data_ptr())
        assert np.array_equal(one_step(s1), ref)
    gpu_ctx.profile(True, timeline=True)
    s1.factorize(Z.data_ptr())
    gpu_ctx.synchronize()
    spans = gpu_ctx.profile_timeline()
    gpu_ctx.profile(False)
    assert np.array_equal(one_step(s1), ref)
    s1.close()
    assert sum(1 for sp in spans if sp[0] == 3) == -(-n // 64)


def test_fp64_fma_peak_is_plausible(gpu_ctx):
    """The FP64 roofline denominator: a B200's 148 SMs at up to ~2 GHz give a
    few tens of TFLOP/s of FP64 FMA, far from zero and from tensor rates."""
    t = gpu_ctx.fp64_fma_peak()
    assert 5.0 < t < 200.0
    # the FP64 tensor cores of a B200 run at about the FMA rate
    tm = gpu_ctx.fp64_mma_peak()
    assert 0.5 * t < tm < 4.0 * t
