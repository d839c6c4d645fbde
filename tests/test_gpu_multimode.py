"""GPU parity of the multimode (M > 1) stepper against the FP64 oracle.

Hermite-Gauss problems (overlap tensor from the mode profiles, per-mode
dispersion by mode group) at the oracle-sized shapes, the config-2 shape
(M = 6, Nt = 2^12 over 5 ps, 1 m, 2 nJ) against the oracle, and the
config-4 shape (M = 10, Nt = 2^14, 2 m, 5 nJ, 64 per-mode phase candidates)
through size-independent properties (the same answer alone and in the
batch, the gradient against central differences of FP64 GPU forwards), and
both configs' forward + adjoint gradients against golden fixtures of the
FP64 oracle (tests/golden/make_multimode_fixtures.py).

Tolerances: field relative L2 ≤ 1e-5 (FP32 mode) and ≤ 1e-10 (FP64 mode),
Raman band fraction within 0.01 dB, gradient ≤ 1e-3 relative.
"""
import os
import sys

import numpy as np
import pytest

from fiberlab_gpu import problem as P
from fiberlab_gpu._capi import FiberLabGPUError, GPUProblem
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)
import make_multimode_fixtures as MF  # noqa: E402  (the fixtures' problem definitions)

pytestmark = pytest.mark.gpu

FIELD_TOL_FP32 = 1e-5
FIELD_TOL_FP64 = 1e-10
GRAD_TOL = 1e-3
DB_TOL = 0.01


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def hg_problem(M, nt, T=5.0, L=0.3, energy=2e-9, seed=0, thz=-5.0, **kw):
    """HG problem with M modes: the first M of the HG(m+n <= order) set."""
    order = {2: 1, 3: 1, 4: 2, 5: 2, 6: 2, 7: 3, 8: 3, 9: 3, 10: 3}[M]
    fp = P.multimode_problem(order, 32, nt, T, L, energy, 200e-15, seed,
                             raman_threshold_thz=thz, **kw)
    if fp.M != M:
        g = fp.gamma[:M, :M, :M, :M].copy()
        u = fp.uw0[:M] * np.sqrt(np.sum(np.abs(fp.uw0) ** 2) / np.sum(np.abs(fp.uw0[:M]) ** 2))
        sim = dict(fp.sim, M=M)
        fp = P.FiberProblem(sim=sim, D=fp.D[:M].copy(), gamma=g, hR=fp.hR, one_m_fR=fp.one_m_fR,
                            L=fp.L, uw0=u, reltol=fp.reltol, abstol=fp.abstol, mask=fp.mask,
                            meta=fp.meta)
    return fp


# M = 6, 8, 10 (Gram ranks 15, 22, 28) take the low-rank form in FP32 mode;
# M = 7, 9 (ranks 19 of 28, 25 of 45: too high for its tables) the full one
@pytest.mark.parametrize("M,nt", [(2, 256), (3, 512), (6, 1024), (7, 256), (8, 256), (9, 256),
                                  (10, 256)])
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_mm_rhs_matches_oracle(gpu_ctx, M, nt, precision):
    fp = hg_problem(M, nt, energy=5e-9)
    rng = np.random.default_rng(M * nt)
    u = fp.uw0 * np.exp(0.3j * rng.standard_normal((M, nt)))
    lam = (rng.standard_normal((M, nt)) + 1j * rng.standard_normal((M, nt))) * 1e-3
    gp = GPUProblem(gpu_ctx, fp, precision)
    z = 0.1234
    tol = 2e-6 if precision == "fp32" else FIELD_TOL_FP64
    assert rel(gp.rhs(z, u), O.rhs_forward(fp, z, u)) < tol
    # with an FP32 forward and M >= 6 the adjoint runs mixed: λ and its
    # transforms in FP64, the forward field's transform and pair products in
    # FP32 (the accuracy that field has) and the per-point contractions on
    # the tensor cores in 3xTF32
    atol = 2e-6 if precision == "fp32" and M >= 6 else FIELD_TOL_FP64
    assert rel(gp.rhs(z, lam, u), O.rhs_adjoint(fp, z, lam, u)) < atol


def test_mm_nonsymmetric_gamma_forward_only(gpu_ctx):
    # test_propagation.jl:178-192: a nonsymmetric γ propagates forward but the
    # adjoint is rejected
    fp = hg_problem(3, 256)
    g = fp.gamma.copy()
    g[0, 0, 1, 1] *= 1.3  # ∫ψ0²ψ1² ≠ 0; γ[0,1,0,1] keeps its value
    fp.gamma = g
    z = 0.05
    rng = np.random.default_rng(5)
    u = fp.uw0 * np.exp(0.2j * rng.standard_normal((3, 256)))
    gp = GPUProblem(gpu_ctx, fp, "fp64")
    assert rel(gp.rhs(z, u), O.rhs_forward(fp, z, u)) < FIELD_TOL_FP64
    with pytest.raises(FiberLabGPUError) as e:
        gp.rhs(z, u, u)
    assert e.value.status == 6


@pytest.mark.parametrize("M,nt", [(3, 512), (6, 1024)])
def test_mm_forward_matches_oracle(gpu_ctx, M, nt):
    fp = hg_problem(M, nt, L=0.5, energy=4e-9)
    zs = [0.0, 0.17, 0.5]
    out, st = GPUProblem(gpu_ctx, fp).forward(saveat=zs)
    ref, rst, _ = O.forward(fp, zsave=zs)
    for i in range(len(zs)):
        assert rel(out[i], ref[i]) < FIELD_TOL_FP32
    assert st["status"] == 0 and st["z_end"] == fp.L
    assert st["nf"] == 3 + 6 * (st["naccept"] + st["nreject"])
    out64, st64 = GPUProblem(gpu_ctx, fp, "fp64").forward(saveat=zs)
    assert rel(out64[-1], ref[-1]) < FIELD_TOL_FP64
    assert st64["naccept"] == rst["naccept"]


def test_mm_config2_shape(gpu_ctx):
    # M = 6 HG(m+n<=2) on a 64x64 grid, Nt = 2^12 over 5 ps, L = 1 m, 2 nJ
    # 200 fs sech², Dirichlet(1) launch weights with random phases.  The band
    # for the 0.01 dB check is the red side beyond 2 THz: at this energy the
    # -13 THz band holds only round-off (J ~ 1e-13)
    fp = P.multimode_problem(2, 64, 4096, 5.0, 1.0, 2e-9, 200e-15, seed=0,
                             raman_threshold_thz=-2.0)
    out, st = GPUProblem(gpu_ctx, fp).forward()
    ref, rst, _ = O.forward(fp)
    assert rel(out[-1], ref[-1]) < FIELD_TOL_FP32
    Jg = P.band_cost_and_seed(out[-1], fp.mask)[0]
    Jo = P.band_cost_and_seed(ref[-1], fp.mask)[0]
    assert abs(10 * np.log10(Jg) - 10 * np.log10(Jo)) < DB_TOL
    n0, n1 = P.photon_number(out[0], fp.sim), P.photon_number(out[-1], fp.sim)
    assert abs(n1 / n0 - 1) < 1e-4


def test_mm_seeded_adjoint_matches_oracle(gpu_ctx):
    fp = hg_problem(3, 512, L=0.4, energy=4e-9)
    gp = GPUProblem(gpu_ctx, fp)
    gp.forward()
    ref, _, dense = O.forward(fp, keep_dense=True)
    seed = ref[-1] * np.linspace(0.2, 1.8, fp.nt)[None, :]
    lam0, st = gp.adjoint(seed)
    lref, _ = O.adjoint(fp, dense, seed)
    assert rel(lam0, lref) < GRAD_TOL
    assert st["adj_naccept"] > 0


def test_mm_band_gradient_shared_phase(gpu_ctx):
    fp = hg_problem(3, 512, L=0.5, energy=6e-9)
    phi = 0.5 * np.random.default_rng(0).standard_normal(fp.nt)
    J, g, st = GPUProblem(gpu_ctx, fp).phase_gradient_batch(phi[None, :])
    Jo, go, _ = O.phase_gradient(fp, phi)
    assert abs(10 * np.log10(J[0]) - 10 * np.log10(Jo)) < DB_TOL
    assert rel(g[0], go) < GRAD_TOL


def _oracle_mode_gradient(fp, phases):
    """∂J/∂φ[m, t] of the band objective from the oracle forward + adjoint
    (physics_models.jl:1042 without the mode sum)."""
    us = fp.uw0 * np.exp(1j * phases)
    out, _, dense = O.forward(fp, u0=us, keep_dense=True)
    J, seed = P.band_cost_and_seed(out[-1], fp.mask)
    lam0, _ = O.adjoint(fp, dense, seed)
    return J, 2 * np.real(np.conj(lam0) * 1j * us)


def test_mm_band_gradient_per_mode_phase(gpu_ctx):
    fp = hg_problem(3, 512, L=0.5, energy=6e-9)
    rng = np.random.default_rng(11)
    phases = rng.standard_normal((2, 3, fp.nt))
    J, g, _ = GPUProblem(gpu_ctx, fp).mode_phase_gradient_batch(phases)
    for b in range(2):
        Jo, go = _oracle_mode_gradient(fp, phases[b])
        assert abs(10 * np.log10(J[b]) - 10 * np.log10(Jo)) < DB_TOL
        assert rel(g[b], go) < GRAD_TOL


def test_mm_gradient_central_differences(gpu_ctx):
    fp = hg_problem(3, 256, L=0.5, energy=6e-9)
    rng = np.random.default_rng(3)
    phases = 0.5 * rng.standard_normal((3, fp.nt))
    J, g, _ = GPUProblem(gpu_ctx, fp).mode_phase_gradient_batch(phases[None])
    gp64 = GPUProblem(gpu_ctx, fp, "fp64")

    def cost(ph):
        out, _ = gp64.forward(fp.uw0 * np.exp(1j * ph))
        return P.band_cost_and_seed(out[-1], fp.mask)[0]
    for _ in range(8):
        d = rng.standard_normal((3, fp.nt))
        d /= np.linalg.norm(d)
        h = 1e-4
        fd = (cost(phases + h * d) - cost(phases - h * d)) / (2 * h)
        assert abs(fd - np.sum(g[0] * d)) <= GRAD_TOL * abs(fd) + 1e-12


def test_mm_config4_shape_properties(gpu_ctx):
    # M = 10 HG(m+n<=3) on a 96x96 grid, Nt = 2^14 over 10 ps, L = 2 m, 5 nJ,
    # 64 per-mode phase candidates φ ~ N(0, 1) run as one batch.  Checked on
    # 4 candidates: alone against the batch (bit-identical), and the FP32
    # gradient against the FP64-mode gradient of the same candidate (the
    # oracle-validated algorithm in FP64; the CPU oracle itself would take
    # tens of minutes per candidate at this size).  The band is the red side
    # beyond 2 THz (J ~ 1e-2).
    fp = P.multimode_problem(3, 96, 16384, 10.0, 2.0, 5e-9, 200e-15, seed=0,
                             raman_threshold_thz=-2.0)
    assert fp.M == 10
    rng = np.random.default_rng(4)
    phases = rng.standard_normal((64, 10, fp.nt))
    J, g, st = GPUProblem(gpu_ctx, fp).mode_phase_gradient_batch(phases)
    assert all(s["status"] == 0 for s in st)
    pick = [0, 21, 42, 63]
    J64, g64, _ = GPUProblem(gpu_ctx, fp, "fp64").mode_phase_gradient_batch(phases[pick])
    for n, b in enumerate(pick):
        Ja, ga, _ = GPUProblem(gpu_ctx, fp).mode_phase_gradient_batch(phases[b:b + 1])
        assert Ja[0] == J[b] and np.array_equal(ga[0], g[b])
        assert abs(10 * np.log10(J[b]) - 10 * np.log10(J64[n])) < DB_TOL
        assert rel(g[b], g64[n]) < GRAD_TOL


def test_mm_config4_gradient_central_differences(gpu_ctx):
    # The adjoint gradient against central differences (h = 1e-4) on the
    # config-4 shape along 4 random unit directions (no bias toward the
    # gradient), both in FP64 mode at tight tolerances (reltol 1e-10,
    # abstol 1e-9): at the default tolerances the two sides differ by their
    # integration error (1e-4 .. 1e-3 on this 10-mode, 2 m problem), which
    # is not what the check is after.  The 8 FD costs run as one batch.
    fp = P.multimode_problem(3, 96, 16384, 10.0, 2.0, 5e-9, 200e-15, seed=0,
                             raman_threshold_thz=-2.0, reltol=1e-10, abstol=1e-9)
    rng = np.random.default_rng(44)
    ph = rng.standard_normal((10, fp.nt))
    gp64 = GPUProblem(gpu_ctx, fp, "fp64")
    J, g, _ = gp64.mode_phase_gradient_batch(ph[None])
    d = rng.standard_normal((4, 10, fp.nt))
    d /= np.linalg.norm(d.reshape(4, -1), axis=1)[:, None, None]
    h = 1e-4
    Jp, _, _ = gp64.mode_phase_gradient_batch(np.concatenate([ph + h * d, ph - h * d]))
    fd = (Jp[:4] - Jp[4:]) / (2 * h)
    ad = np.einsum("bmt,mt->b", d, g[0])
    err = np.abs(fd - ad) / np.abs(fd)
    assert np.all(err <= GRAD_TOL), (err, fd, ad)


def test_mm_config2_against_oracle_fixture(gpu_ctx):
    # config 2 (M = 6, Nt = 2^12 over 5 ps, 1 m, 2 nJ, Dirichlet(1) launch):
    # FP32 forward + adjoint with per-mode phases N(0, 0.5²) against the FP64
    # oracle's output field, band fraction and per-mode gradient
    # (a dense-output buffer that holds the whole solve: the adjoint runs
    # 0 <- L without checkpoint stops, as the oracle's does)
    from fiberlab_gpu._capi import Context
    fx = np.load(os.path.join(GOLDEN, "mm_config2.npz"))
    fp = MF.config2_problem()
    ph = MF.config2_phases(fp)
    gp = GPUProblem(Context(0, segment_steps=128), fp)
    out, st = gp.forward(fp.uw0 * np.exp(1j * ph))
    assert rel(out[-1], fx["uL"]) < FIELD_TOL_FP32
    J, g, gst = gp.mode_phase_gradient_batch(ph[None])
    assert gst[0]["status"] == 0 and gst[0]["recompute_steps"] == 0
    assert abs(10 * np.log10(J[0]) - 10 * np.log10(float(fx["J"]))) < DB_TOL
    assert rel(g[0], fx["grad"]) < GRAD_TOL, rel(g[0], fx["grad"])


def test_mm_config4_against_oracle_fixture(gpu_ctx):
    # config 4 (M = 10, Nt = 2^14 over 10 ps, 2 m, 5 nJ): 4 per-mode phase
    # candidates N(0, 1) as one FP32 batch against the FP64 oracle's band
    # fractions and gradients (on the bins where the launch is not
    # negligible: the gradient vanishes with it), and candidate 0's field
    from fiberlab_gpu._capi import Context
    fx = np.load(os.path.join(GOLDEN, "mm_config4.npz"))
    fp = MF.config4_problem()
    seeds = [int(x) for x in fx["seeds"]]
    phs = np.stack([MF.config4_phases(fp, s) for s in seeds])
    gp = GPUProblem(Context(0, segment_steps=160), fp)
    J, g, st = gp.mode_phase_gradient_batch(phs)
    idx = fx["idx"]
    for b in range(len(seeds)):
        assert st[b]["status"] == 0 and st[b]["recompute_steps"] == 0
        assert abs(10 * np.log10(J[b]) - 10 * np.log10(float(fx["J"][b]))) < DB_TOL
        go = fx["grad"][b].astype(np.float64)
        outside = np.ones(fp.nt, bool)
        outside[idx] = False
        e = np.sqrt(np.sum((g[b][:, idx] - go) ** 2) + np.sum(g[b][:, outside] ** 2))
        assert e / np.linalg.norm(go) < GRAD_TOL, (b, e / np.linalg.norm(go))
    out, _ = gp.forward(fp.uw0 * np.exp(1j * phs[0]))
    assert rel(out[-1], fx["uL0"].astype(np.complex128)) < FIELD_TOL_FP32


def test_mm_adjoint_beyond_checkpoint_capacity(gpu_ctx):
    # the multimode stepper replays each checkpoint segment once per
    # sub-segment when a solve has more accepted steps than checkpoints x
    # segment_steps
    from fiberlab_gpu._capi import Context
    fp = hg_problem(3, 256, L=0.5, energy=6e-9)
    phi = 0.5 * np.random.default_rng(32).standard_normal(fp.nt)
    J, g, st = GPUProblem(Context(0, checkpoints=2, segment_steps=3), fp).phase_gradient_batch(
        phi[None, :])
    assert st[0]["status"] == 0 and st[0]["naccept"] > 6
    Jo, go, _ = O.phase_gradient(fp, phi)
    assert abs(10 * np.log10(J[0]) - 10 * np.log10(Jo)) < DB_TOL
    assert rel(g[0], go) < GRAD_TOL


def test_mm_save_on_interior_step_end(gpu_ctx):
    # the multimode stepper's dense output at a save position exactly on an
    # interior accepted step end (sol.t from a first forward)
    fp = hg_problem(3, 256, L=0.5, energy=6e-9)
    gp = GPUProblem(gpu_ctx, fp)
    gp.forward()
    t = gp.forward_times()
    assert t[0] == 0.0 and t[-1] == fp.L and np.all(np.diff(t) > 0)
    zk = float(t[len(t) // 2])
    zs = [0.0, np.nextafter(zk, 0.0), zk, np.nextafter(zk, 1.0), fp.L]
    out, st = gp.forward(saveat=zs)
    np.testing.assert_array_equal(gp.forward_times(), t)
    ref, _, _ = O.forward(fp, zsave=zs)
    for i in range(len(zs)):
        assert rel(out[i], ref[i]) < FIELD_TOL_FP32, (i, rel(out[i], ref[i]))
    assert rel(out[1], out[2]) < 1e-6 and rel(out[3], out[2]) < 1e-6


def test_mm_grin_fiber_forward(gpu_ctx):
    # a 3-mode parabolic GRIN fiber from the host mode solver
    # (fibers.jl:91-132) through the multimode GPU stepper against the oracle
    from fiberlab_gpu import grin as G
    fp = G.grin_problem(3, 512, 5.0, 0.3, 4e-9, 200e-15, nx=48, weights=[0.8, 0.5, 0.33],
                        raman_threshold_thz=-5.0)
    out, st = GPUProblem(gpu_ctx, fp).forward()
    ref, _, _ = O.forward(fp)
    assert st["status"] == 0
    assert rel(out[-1], ref[-1]) < FIELD_TOL_FP32


@pytest.mark.parametrize("objective", ["fundamental_mode", "worst_mode", "raman_peak"])
@pytest.mark.parametrize("log_cost", [False, True])
def test_mm_device_objective_seeds(gpu_ctx, objective, log_cost):
    # multimode device seeds (fl_problem_set_objective) against the oracle's
    # forward and adjoint with the host seed of the same objective
    from fiberlab_gpu import objectives as Ob
    fp = hg_problem(3, 512, L=0.5, energy=6e-9)
    phi = 0.5 * np.random.default_rng(12).standard_normal(fp.nt)
    gp = GPUProblem(gpu_ctx, fp)
    gp.set_objective(objective, 20.0)
    J, g, _ = gp.phase_gradient_batch(phi[None, :], log_cost=log_cost)
    shaped = fp.uw0 * np.exp(1j * phi)[None, :]
    out, _, dense = O.forward(fp, u0=shaped, keep_dense=True)
    Jo, seed = Ob.cost_and_seed(objective, out[-1], fp.mask, fp.sim, log_cost, worst_mode_tau=20.0)
    lam0, _ = O.adjoint(fp, dense, seed)
    go = (2 * np.real(np.conj(lam0) * 1j * shaped)).sum(axis=0)
    if log_cost:
        assert abs(J[0] - Jo) < DB_TOL
    else:
        assert abs(J[0] - Jo) <= 1e-4 * abs(Jo)
    assert rel(g[0], go) < GRAD_TOL
