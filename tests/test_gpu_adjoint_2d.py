"""GPU parity of the FWI gradient and RTM image drivers (through the C ABI).

Exact arithmetic with lossless checkpoints must reproduce the oracle's
FwiAcoustic2D::run_optimal / RtmAcoustic2D::run_optimal outputs bit for bit,
for any Revolve snapshot count (recomputation from checkpoints is exact) and
for several shots with different windows batched in one run.  The production
settings (FMA arithmetic, FP64 accumulation, FP16/BF16 checkpoints) are held to
relative-L2 bounds against the FP64 GPU propagator.
"""
import numpy as np
import pytest

from rockseis_b200 import abi
from rockseis_b200.rockseis import AdjointBatch, Data2D, FwiAcoustic2D, Image2D, RtmAcoustic2D, fwi_gradient_batch
from tests.cases import fwi_case, oracle_fwi, oracle_rtm, rel_l2

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-5       # plain FP32 bar of the gradient against the exact result
CKPT16_TOL = 1e-3     # FP16-checkpoint bar against the FP64 propagator


def make_fwi(c, precision=None, ncheck=5, ckpt=abi.CKPT_NATIVE, accum=abi.ACCUM_REFERENCE):
    prec = c.precision if precision is None else precision
    c.rec.data = np.ascontiguousarray(c.obs.astype(abi.real_dtype(prec)))
    f = FwiAcoustic2D(c.model, c.src, c.rec, c.order, 1, precision=prec)
    f.setNcheck(ncheck)
    f.setCheckpointPrecision(ckpt)
    f.setAccumulation(accum)
    f.setVpgrad(Image2D("vpgrad", c.model, 1, 1, prec))
    f.setRhograd(Image2D("rhograd", c.model, 1, 1, prec))
    t = abi.real_dtype(prec)
    w = Data2D(c.src.ntrace, c.nt, c.dt, 0.0, prec)
    dm = Data2D(c.rec.ntrace, c.nt, c.dt, 0.0, prec)
    dr = Data2D(c.rec.ntrace, c.nt, c.dt, 0.0, prec)
    f.setWavgrad(w)
    f.setDatamodP(dm)
    f.setDataresP(dr)
    assert w.data.dtype == t
    return f


def outputs(f):
    return dict(vpgrad=f.vpgrad.getImagedata()[0, 0], rhograd=f.rhograd.getImagedata()[0, 0], wavgrad=f.wavgrad.data,
                datamod=f.datamodP.data, datares=f.dataresP.data, misfit=f.getMisfit())


def assert_same(got, ref):
    for k in ("vpgrad", "rhograd", "wavgrad", "datamod", "datares"):
        assert np.abs(ref[k]).max() > 0, k
        assert np.array_equal(got[k], ref[k]), f"{k}: max abs diff {np.abs(got[k] - ref[k]).max()}"
    assert got["misfit"] == ref["misfit"]


@pytest.mark.parametrize("ncheck", [4, 300])
def test_fwi_source_illumination_equals_reference(require_gpu, ncheck):
    # FwiAcoustic2D::setSrcilum: srcilum -= (-2/vp) Pfw^2 inside crossCorr, checked against
    # the reference library itself together with every other output
    from oracle import api
    if not api.ref_available():
        pytest.skip("reference library oracle/_ref not built")
    c = fwi_case()
    ref = api.ref_fwi_a2d(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords, c.obs, ncheck,
                          srcilum=True)
    f = make_fwi(c, ncheck=ncheck)
    f.setSrcilum(Image2D("srcilum", c.model, 1, 1, c.precision))
    assert f.run_optimal() == 1
    assert_same(outputs(f), ref)
    il = f.srcilum.getImagedata()[0, 0]
    assert np.abs(ref["srcilum"]).max() > 0
    assert np.array_equal(il, ref["srcilum"]), f"srcilum: max abs diff {np.abs(il - ref['srcilum']).max()}"


def test_fwi_source_illumination_batched_fp64_accumulation(require_gpu):
    # batched windows, only the second shot asks for the illumination; FP64 accumulation
    # against the per-shot exact result
    cases = [fwi_case(nx=81, nz=61, seed=1, scoord=(400.3, 23.7)), fwi_case(nx=97, nz=53, seed=2, scoord=(150.9, 31.2))]
    exact = []
    for c in cases:
        f = make_fwi(c, ncheck=6)
        f.setSrcilum(Image2D("srcilum", c.model, 1, 1, c.precision))
        f.run_optimal()
        exact.append(f.srcilum.getImagedata()[0, 0].copy())
    jobs = [make_fwi(c, ncheck=6, accum=abi.ACCUM_F64) for c in cases]
    jobs[1].setSrcilum(Image2D("srcilum", cases[1].model, 1, 1, cases[1].precision))
    fwi_gradient_batch(jobs)
    assert jobs[0].srcilum is None
    assert rel_l2(jobs[1].srcilum.getImagedata()[0, 0], exact[1]) < 1e-6


@pytest.mark.parametrize("ncheck", [2, 5, 17, 300])
def test_fwi_gradient_exact_bitwise(require_gpu, ncheck):
    c = fwi_case()
    ref = oracle_fwi(c)
    f = make_fwi(c, ncheck=ncheck)
    assert f.run_optimal() == 1
    assert_same(outputs(f), ref)


def test_fwi_gradient_free_surface_and_off_grid_receiver(require_gpu):
    c = fwi_case(fs=1, nrec=33, rx0=-17.0)          # first receiver off the grid
    assert (c.rec.gmap[:, 0] < 0).any()
    ref = oracle_fwi(c)
    f = make_fwi(c, ncheck=9)
    f.run_optimal()
    assert_same(outputs(f), ref)


def test_fwi_gradient_batched_windows_bitwise(require_gpu):
    cases = [fwi_case(nx=81, nz=61, seed=1, scoord=(400.3, 23.7)),
             fwi_case(nx=97, nz=53, seed=2, scoord=(150.9, 31.2)),
             fwi_case(nx=64, nz=70, seed=3, scoord=(322.0, 12.5))]
    refs = [oracle_fwi(c) for c in cases]
    jobs = [make_fwi(c, ncheck=6) for c in cases]
    assert fwi_gradient_batch(jobs) == 1
    for f, ref in zip(jobs, refs):
        assert_same(outputs(f), ref)


def test_fwi_resident_batch_runs_repeat(require_gpu):
    c = fwi_case(nt=200)
    ref = oracle_fwi(c)
    f = make_fwi(c, ncheck=8)
    b = AdjointBatch([f])
    for _ in range(2):
        for img in (f.vpgrad, f.rhograd):
            img.getImagedata()[:] = 0
        for d in (f.wavgrad, f.datamodP, f.dataresP):
            d.data[:] = 0
        f.misfit = 0.0
        b.run()
        b.read()
        assert_same(outputs(f), ref)
    st = b.stats()
    assert st["bw_steps"] == c.nt - 1
    # Revolve's advances plus the forward step taken at FIRSTURN
    assert st["fw_steps"] == abi.lib.rsgpu_revolve_numforw(c.nt, 8) + 1
    b.close()


@pytest.mark.parametrize("nhx,nhz", [(1, 1), (3, 1), (1, 3), (5, 3)])
def test_rtm_image_exact_bitwise(require_gpu, nhx, nhz):
    c = fwi_case(nt=250)
    ref = oracle_rtm(c, c.obs, nhx, nhz)
    c.rec.data = np.ascontiguousarray(c.obs)
    img = Image2D("pimage", c.model, nhx, nhz)
    r = RtmAcoustic2D(c.model, img, c.src, c.rec, c.order, 1)
    r.setNcheck(7)
    assert r.run_optimal() == 1
    got = img.getImagedata()
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), f"max abs diff {np.abs(got - ref).max()}"


GRAD = ("vpgrad", "rhograd", "wavgrad")


def _rel(got, ref, keys=GRAD):
    return {k: rel_l2(got[k], ref[k]) for k in keys}


@pytest.fixture(scope="module")
def fp64_and_exact():
    """FP64 GPU propagator (the precision yardstick) and the reference-exact float result."""
    c64 = fwi_case(precision=abi.F64)
    f64 = make_fwi(c64, ncheck=10, accum=abi.ACCUM_F64)
    f64.run_optimal()
    c = fwi_case()
    return outputs(f64), oracle_fwi(c)


def test_fp64_propagator_against_reference_float(require_gpu, fp64_and_exact):
    # the reference's own float arithmetic sits ~1e-4..1e-3 from FP64 here: the
    # residual is ~1% of the data, so its relative rounding error is ~100x the
    # gather's (which agrees to ~1e-6)
    ref64, exact = fp64_and_exact
    assert rel_l2(exact["datamod"], ref64["datamod"]) <= 1e-5
    err = _rel(exact, ref64)
    print(f"reference float arithmetic vs FP64: {err}")
    assert max(err.values()) <= 1e-3


@pytest.mark.parametrize("accum", [abi.ACCUM_REFERENCE, abi.ACCUM_F64])
def test_fwi_fast_mode_as_accurate_as_reference_float(require_gpu, fp64_and_exact, accum):
    ref64, exact = fp64_and_exact
    c = fwi_case()
    f = make_fwi(c, precision=abi.F32_FAST, ncheck=10, accum=accum)
    f.run_optimal()
    got = outputs(f)
    # modelled data: plain FP32 bar against the exact float path
    assert rel_l2(got["datamod"], exact["datamod"]) <= FAST_TOL
    err, base = _rel(got, ref64), _rel(exact, ref64)
    print(f"FMA arithmetic vs FP64: {err} (reference float: {base})")
    for k in GRAD:
        assert err[k] <= 1.25 * base[k] + 1e-5, k
    assert abs(got["misfit"] - ref64["misfit"]) <= 1e-4 * abs(ref64["misfit"])


# Relative L2 of the gradients against the FP64 propagator with 16-bit checkpoints
# (FMA arithmetic, FP64 accumulation): FP16 holds the 1e-3 bar; BF16 (8-bit
# mantissa) is held to 2e-3.
@pytest.mark.parametrize("ckpt,tol", [(abi.CKPT_F16, CKPT16_TOL), (abi.CKPT_BF16, 2e-3)])
def test_fwi_16bit_checkpoints_against_fp64_propagator(require_gpu, fp64_and_exact, ckpt, tol):
    ref64, _ = fp64_and_exact
    c = fwi_case()
    f = make_fwi(c, precision=abi.F32_FAST, ncheck=10, ckpt=ckpt, accum=abi.ACCUM_F64)
    f.run_optimal()
    err = _rel(outputs(f), ref64)
    print(f"checkpoint format {ckpt}: relative L2 against the FP64 propagator {err}")
    assert max(err.values()) <= tol, err


def test_sharded_stack_on_one_rank_equals_sum_of_shots(require_gpu):
    from rockseis_b200.distributed import fwi_gradient_sharded
    cases = [fwi_case(scoord=(sx, 23.7), seed=1) for sx in (150.9, 400.3, 610.2)]
    refs = [oracle_fwi(c) for c in cases]
    jobs = [make_fwi(c, ncheck=6) for c in cases]
    vp, rho, mis = fwi_gradient_sharded(jobs, 0, 1)
    assert vp.shape == jobs[0].vpgrad.getImagedata().shape      # (nhx, nhz, nz, nx) like the images
    assert np.array_equal(vp[0, 0], sum(r["vpgrad"].astype(np.float64) for r in refs))
    assert np.array_equal(rho[0, 0], sum(r["rhograd"].astype(np.float64) for r in refs))
    assert mis == sum(float(r["misfit"]) for r in refs)


@pytest.mark.parametrize("ncheck", [4, 11])
def test_fwi_correlation_misfit_exact_bitwise(require_gpu, ncheck):
    # CORRELATION misfit: per-trace normalised correlation, its residuals and the
    # 97th-percentile residual clip (radix select on the GPU, a sort in the oracle)
    c = fwi_case()
    ref = oracle_fwi(c, misfit=abi.MISFIT_CORRELATION)
    assert (ref["datares"] == 0).mean() >= 0.03
    f = make_fwi(c, ncheck=ncheck)
    f.setMisfit_type(abi.MISFIT_CORRELATION)
    assert f.run_optimal() == 1
    assert_same(outputs(f), ref)


def test_fwi_correlation_batched_windows_bitwise(require_gpu):
    cases = [fwi_case(nx=81, nz=61, seed=1, scoord=(400.3, 23.7), fs=1),
             fwi_case(nx=97, nz=53, seed=2, scoord=(150.9, 31.2), nrec=41, rx0=-17.0),
             fwi_case(nx=64, nz=70, seed=3, scoord=(322.0, 12.5))]
    refs = [oracle_fwi(c, misfit=abi.MISFIT_CORRELATION) for c in cases]
    jobs = [make_fwi(c, ncheck=6) for c in cases]
    for j in jobs:
        j.setMisfit_type(abi.MISFIT_CORRELATION)
    assert fwi_gradient_batch(jobs) == 1
    for f, ref in zip(jobs, refs):
        assert_same(outputs(f), ref)


def test_fwi_correlation_fp64_accumulation_close(require_gpu):
    c = fwi_case()
    ref = oracle_fwi(c, misfit=abi.MISFIT_CORRELATION)
    f = make_fwi(c, ncheck=8, accum=abi.ACCUM_F64)
    f.setMisfit_type(abi.MISFIT_CORRELATION)
    f.run_optimal()
    got = outputs(f)
    assert np.array_equal(got["datares"], ref["datares"])            # residuals do not depend on the accumulator
    assert abs(got["misfit"] - ref["misfit"]) <= 1e-5 * abs(ref["misfit"])
    for k in GRAD:
        assert rel_l2(got[k], ref[k]) <= 1e-5, k


# ---------------------------------------------------------------- FULL snapshots (FwiAcoustic2D::run, RtmAcoustic2D::run)
def _snapfull():
    import os
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "snapfull.npz"))


def full_reference(c, snapinc, noreverse=0):
    """FwiAcoustic2D::run of the reference: the library itself where oracle/_ref is
    built, else the committed outputs (tests/golden/make_golden_snapfull.py)."""
    from oracle import api
    if api.ref_available():
        return api.ref_fwi_a2d_full(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords,
                                    c.obs.astype(np.float32), snapinc, noreverse=noreverse)
    g = _snapfull()
    if f"fwi_s{snapinc}_vpgrad" not in g.files and not noreverse:
        pytest.skip(f"no committed outputs for snapinc {snapinc} and the reference library is not built")
    assert np.array_equal(c.obs.astype(np.float32), g["obs"]) and np.array_equal(c.pb.vp, g["vp"])
    out = {k: g[f"fwi_{k}"] for k in ("datamod", "datares")}
    out["misfit"] = float(g["fwi_misfit"])
    for k in ("vpgrad", "rhograd", "wavgrad"):
        out[k] = np.zeros_like(g["fwi_s3_vpgrad"] if k != "wavgrad" else g["fwi_s3_wavgrad"]) if noreverse \
            else g[f"fwi_s{snapinc}_{k}"]
    if noreverse:
        out["datares"] = np.zeros_like(out["datares"])
    return out


@pytest.mark.parametrize("snapinc", [1, 3, 7])
def test_fwi_full_snapshots_bitwise(require_gpu, snapinc):
    # snapinc 3 and 7 leave enddiff = 2 and 5: the adjoint times that correlate are not
    # the forward times that were saved, as in Snapshot2D
    c = fwi_case()
    ref = full_reference(c, snapinc)
    f = make_fwi(c)
    f.setSnapinc(snapinc)
    assert f.run() == 1
    assert_same(outputs(f), ref)


def test_fwi_full_snapshots_noreverse(require_gpu):
    # forward pass, datamodP and the misfit only; gradients, wavelet gradient and
    # residuals stay as the caller left them
    c = fwi_case()
    ref = full_reference(c, 3, noreverse=1)
    f = make_fwi(c)
    f.setSnapinc(3)
    f.setNoreverse(True)
    assert f.run() == 1
    got = outputs(f)
    assert np.abs(ref["datamod"]).max() > 0
    assert np.array_equal(got["datamod"], ref["datamod"])
    assert got["misfit"] == ref["misfit"]
    for k in ("vpgrad", "rhograd", "wavgrad", "datares"):
        assert not np.any(got[k]), k


@pytest.mark.parametrize("snapinc,nhx,nhz", [(4, 3, 1), (1, 1, 1), (5, 1, 3)])
def test_rtm_full_snapshots_bitwise(require_gpu, snapinc, nhx, nhz):
    from oracle import api
    c = fwi_case()
    if api.ref_available():
        ref = api.ref_rtm_a2d_full(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords,
                                   c.obs.astype(np.float32), snapinc, nhx=nhx, nhz=nhz)
    elif (snapinc, nhx, nhz) == (4, 3, 1):
        ref = _snapfull()["rtm_s4_h3"]
    else:
        pytest.skip("reference library not built")
    c.rec.data = np.ascontiguousarray(c.obs)
    img = Image2D("pimage", c.model, nhx, nhz)
    r = RtmAcoustic2D(c.model, img, c.src, c.rec, c.order, snapinc)
    assert r.run() == 1
    got = img.getImagedata()
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), f"max abs diff {np.abs(got - ref).max()}"


def test_fwi_full_snapshots_batched_windows_bitwise(require_gpu):
    from oracle import api
    if not api.ref_available():
        pytest.skip("reference library not built")
    cases = [fwi_case(nx=81, nz=61, seed=1, scoord=(400.3, 23.7)), fwi_case(nx=97, nz=53, seed=2, scoord=(150.9, 31.2))]
    refs = [full_reference(c, 5) for c in cases]
    jobs = [make_fwi(c) for c in cases]
    for j in jobs:
        j.setSnapinc(5)
    assert fwi_gradient_batch(jobs, snapmethod=abi.SNAP_FULL) == 1
    for j, ref in zip(jobs, refs):
        assert_same(outputs(j), ref)


@pytest.mark.parametrize("ckpt", [abi.CKPT_F16, abi.CKPT_BF16])
def test_fwi_full_16bit_snapshots_close(require_gpu, ckpt):
    # 16-bit snapshots with a power-of-two scale per shot: the same bars as the
    # 16-bit Revolve checkpoints hold against the lossless result
    c = fwi_case()
    ref = full_reference(c, 3)
    f = make_fwi(c, ckpt=ckpt)
    f.setSnapinc(3)
    assert f.run() == 1
    got = outputs(f)
    tol = CKPT16_TOL if ckpt == abi.CKPT_F16 else 3e-3
    for k in GRAD:
        assert rel_l2(got[k], ref[k]) < tol, (k, rel_l2(got[k], ref[k]))
    assert np.array_equal(got["datamod"], ref["datamod"])


# ---------------------------------------------------------------- ADAPTIVE misfits (Wiener shaping filters)
def adaptive_reference(c, misfit, ncheck=7, dims="a2d"):
    """FwiAcoustic2D::run_optimal with an ADAPTIVE misfit: the reference library where
    oracle/_ref is built, else the committed outputs (tests/golden/make_golden_adaptive.py)."""
    import os
    from oracle import api
    if api.ref_available():
        return api.ref_fwi_a2d(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords,
                               c.obs.astype(np.float32), ncheck, misfit=misfit)
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "adaptive.npz"))
    assert ncheck == 7 and np.array_equal(c.obs.astype(np.float32), g[f"{dims}_obs"])
    name = {abi.MISFIT_ADAPTIVE_GAUSS: "gauss", abi.MISFIT_ADAPTIVE_LINEAR: "linear"}[misfit]
    out = {k: g[f"{dims}_{name}_{k}"] for k in ("vpgrad", "rhograd", "wavgrad", "datares")}
    out["datamod"] = g[f"{dims}_datamod"]
    out["misfit"] = float(g[f"{dims}_{name}_misfit"])
    return out


@pytest.mark.parametrize("misfit", [abi.MISFIT_ADAPTIVE_GAUSS, abi.MISFIT_ADAPTIVE_LINEAR])
def test_fwi_adaptive_misfit_bitwise(require_gpu, misfit):
    # shaping filters by Levinson recursion, SU-ordered correlations and convolution,
    # the 97th-percentile residual clip: every output equal to the reference's
    c = fwi_case()
    ref = adaptive_reference(c, misfit)
    f = make_fwi(c, ncheck=7)
    f.setMisfit_type(misfit)
    assert f.run_optimal() == 1
    got = outputs(f)
    assert_same(got, ref)
    assert (got["misfit"] < 0) == (misfit == abi.MISFIT_ADAPTIVE_GAUSS)
    assert (got["datares"] == 0).mean() >= 0.03


def test_fwi_adaptive_misfit_batched_windows_bitwise(require_gpu):
    from oracle import api
    if not api.ref_available():
        pytest.skip("reference library not built")
    cases = [fwi_case(nx=81, nz=61, seed=1, scoord=(400.3, 23.7)), fwi_case(nx=97, nz=53, seed=2, scoord=(150.9, 31.2))]
    refs = [adaptive_reference(c, abi.MISFIT_ADAPTIVE_LINEAR, ncheck=6) for c in cases]
    jobs = [make_fwi(c, ncheck=6) for c in cases]
    for j in jobs:
        j.setMisfit_type(abi.MISFIT_ADAPTIVE_LINEAR)
    assert fwi_gradient_batch(jobs) == 1
    for j, ref in zip(jobs, refs):
        assert_same(outputs(j), ref)


def test_fwi_adaptive_misfit_fp64_accumulation_close(require_gpu):
    c = fwi_case()
    ref = adaptive_reference(c, abi.MISFIT_ADAPTIVE_GAUSS)
    f = make_fwi(c, ncheck=7, accum=abi.ACCUM_F64)
    f.setMisfit_type(abi.MISFIT_ADAPTIVE_GAUSS)
    assert f.run_optimal() == 1
    got = outputs(f)
    for k in GRAD:
        assert rel_l2(got[k], ref[k]) < 1e-5, (k, rel_l2(got[k], ref[k]))
    assert abs(got["misfit"] - ref["misfit"]) <= 1e-5 * abs(ref["misfit"])


@pytest.mark.parametrize("snapinc,nhx", [(1, 1), (3, 1), (4, 3)])
def test_rtm_edge_snapshots_bitwise(require_gpu, snapinc, nhx):
    # RtmAcoustic2D::run_edge: the four edge lines of P saved every snapinc steps; the
    # source wavefield is stepped again from zero with the saved lines written back in
    from oracle import api
    c = fwi_case()
    if api.ref_available():
        ref = api.ref_rtm_a2d_full(c.pb, c.src.scoords, c.src.data.astype(np.float32), c.rec.gcoords,
                                   c.obs.astype(np.float32), snapinc, nhx=nhx, edges=True)
    elif (snapinc, nhx) == (4, 3):
        ref = _snapfull()["rtm_edge_s4_h3"]
    else:
        pytest.skip("reference library not built")
    c.rec.data = np.ascontiguousarray(c.obs)
    img = Image2D("pimage", c.model, nhx, 1)
    r = RtmAcoustic2D(c.model, img, c.src, c.rec, c.order, snapinc)
    assert r.run_edge() == 1
    got = img.getImagedata()
    assert np.abs(ref).max() > 0
    assert np.array_equal(got, ref), f"max abs diff {np.abs(got - ref).max()}"
