"""GPU parity of the adjoint of the H_eff contraction (dE/dlambda for a vertex
coupling lambda, W = W0 + lambda dW), through the C ABI.

* H_eff level: for a fixed wavefunction, E(lambda) = <x|H_eff(W0 + lambda dW)|x>
  / <x|x> is quadratic in lambda (H_eff is bilinear in the two vertex MPOs),
  so the central difference (E(+1) - E(-1)) / 2 is its exact derivative at 0.
  It is taken with the oracle's block-sparse matvec; the GPU adjoint must
  agree to 1e-10 relative, also with environment derivatives dL, dR added
  (E is linear in each environment).
* iDMRG level: with no truncation the grown state is the exact ground state
  of the open 2N-vertex chain, so dE_N/dlambda (Hellmann-Feynman, with the
  derivative environments carried through the growth) must equal the
  central difference of the grown energies at lambda +- 1e-4 to 1e-6
  relative (the difference quotient's own error is ~1e-8)."""
import numpy as np
import pytest

from oracle import blocks as ob

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from chainamps_b200 import Context
    c = Context(0)
    yield c
    c.close()


def env_mats(t, chi, D):
    """Dense [a', a] blocks per MPO slot of an environment tensor (None if zero)."""
    M = np.zeros((chi, D * chi), np.complex128)
    cols = np.repeat(np.arange(t.cols), np.diff(t.colptr))
    M[t.rowind, cols] = t.values
    T = M.reshape(chi, D, chi, order="F")
    return [T[:, b, :] if np.any(T[:, b, :]) else None for b in range(D)]


def xxz_mpo(jz):
    from chainamps_b200 import models
    return models.xxz_model(1.0, jz, 0.0)


@pytest.mark.parametrize("with_env", [False, True])
def test_heff_adjoint_matches_oracle(ctx, with_env):
    from chainamps_b200 import TwoVertexComponents, models, upload_block
    rules, ch, W0, bq = xxz_mpo(0.7)
    dW = 0.5 * (xxz_mpo(1.7)[2] - xxz_mpo(-0.3)[2])      # dW / dJz (W is affine in Jz)
    D = bq.shape[0]
    used_l = sorted({int(b) for b in np.nonzero(np.any(W0 != 0, axis=(0, 2, 3)))[0]})
    used_r = sorted({int(b) for b in np.nonzero(np.any(W0 != 0, axis=(0, 1, 2)))[0]})
    rng = np.random.default_rng(3)
    bond = models.gaussian_bond(28, step=2, width=3.0)
    chi = bond.shape[0]
    L = models.random_environment(rng, rules, bond, bq, used_l, right=False)
    R = models.random_environment(rng, rules, bond, bq, used_r, right=True)
    dL = models.random_environment(rng, rules, bond, bq, used_l, right=False)
    dR = models.random_environment(rng, rules, bond, bq, used_r, right=True)
    Wt = models.mpo_tensor(ch, W0, bq)
    gpu = TwoVertexComponents(ctx, rules, L, Wt, R)
    x = rng.standard_normal(gpu.n) + 1j * rng.standard_normal(gpu.n)
    gpu.set_theta(x)
    if with_env:
        bl = upload_block(ctx, rules, dL, Wt, right=False)
        br = upload_block(ctx, rules, dR, Wt, right=True)
        g = gpu.adjoint(models.mpo_tensor(ch, dW, bq), bl, br)
    else:
        g = gpu.adjoint(models.mpo_tensor(ch, dW, bq))

    def energy(W, Lt, Rt):
        bh = ob.BlockHeff(rules, ch, bond, bond, bq, W, env_mats(Lt, chi, D), env_mats(Rt, chi, D))
        assert bh.n == gpu.n
        return np.vdot(x, bh.matvec(x)).real / np.vdot(x, x).real
    ref = 0.5 * (energy(W0 + dW, L, R) - energy(W0 - dW, L, R))
    if with_env:
        ref += energy(W0, dL, R) + energy(W0, L, dR)
    assert abs(g - ref) <= 1e-10 * max(1.0, abs(ref)), (g, ref)


def test_adjoint_rejects_pattern_outside_w(ctx):
    from chainamps_b200 import TwoVertexComponents, models, CmpsError
    rules, ch, W0, bq = xxz_mpo(0.0)                       # Jz = 0: no Sz Sz entries in W
    dW = 0.5 * (xxz_mpo(1.0)[2] - xxz_mpo(-1.0)[2])
    used_l = sorted({int(b) for b in np.nonzero(np.any(W0 != 0, axis=(0, 2, 3)))[0]})
    used_r = sorted({int(b) for b in np.nonzero(np.any(W0 != 0, axis=(0, 1, 2)))[0]})
    rng = np.random.default_rng(4)
    bond = models.gaussian_bond(12, step=2, width=2.0)
    L = models.random_environment(rng, rules, bond, bq, used_l, right=False)
    R = models.random_environment(rng, rules, bond, bq, used_r, right=True)
    gpu = TwoVertexComponents(ctx, rules, L, models.mpo_tensor(ch, W0, bq), R)
    gpu.set_theta(np.ones(gpu.n, complex))
    with pytest.raises(CmpsError) as e:
        gpu.adjoint(models.mpo_tensor(ch, dW, bq))
    assert e.value.code == 1


def test_idmrg_gradient_matches_finite_difference(ctx):
    from chainamps_b200 import iDMRG, models, CMPS_FP64, CMPS_SPLIT_TF32
    jz, h = 0.7, 1e-4
    rules, ch, W0, bq = xxz_mpo(jz)
    dW = 0.5 * (xxz_mpo(jz + 1.0)[2] - xxz_mpo(jz - 1.0)[2])
    T = lambda W: models.mpo_tensor(ch, W, bq)
    run = iDMRG(ctx, rules, T(W0), tol=1e-13, krylov_dim=32, gradient=T(dW))
    mixed = iDMRG(ctx, rules, T(W0), precision=CMPS_SPLIT_TF32, tol=1e-13, krylov_dim=32, gradient=T(dW))
    rp = iDMRG(ctx, rules, T(xxz_mpo(jz + h)[2]), tol=1e-13, krylov_dim=32)
    rm = iDMRG(ctx, rules, T(xxz_mpo(jz - h)[2]), tol=1e-13, krylov_dim=32)
    for step in range(5):                                  # bond dimensions 2 .. 32 <= chi: no truncation
        a = run.grow(64, 0.0)
        b = mixed.grow(64, 0.0)
        fd = (rp.grow(64, 0.0)["energy"] - rm.grow(64, 0.0)["energy"]) / (2 * h)
        assert a["truncation"] == 0.0
        assert abs(a["gradient"] - fd) <= 1e-6 * max(1.0, abs(fd)), (step, a["gradient"], fd)
        assert abs(b["gradient"] - a["gradient"]) <= 1e-8 * max(1.0, abs(a["gradient"])), (step, b, a)


@pytest.mark.parametrize("which", ["g", "j_perp"])
def test_coupled_ising_gradients(ctx, which):
    """dE/dg (field, chain basis fixed at g0) and dE/dJ_perp on coupled
    Ising chains (4-site vertices cut to 8 states): the carried iDMRG
    gradient against central differences of the grown energy while the
    bond dimension (8, 64) stays below chi (no truncation)."""
    from chainamps_b200 import iDMRG, models
    g0, jp0, h = 1.2, 0.05, 1e-4

    def mpo(g, jp):
        ch, ops, H, _, _ = models.ising_chain_vertex(4, g, 8, g_basis=g0)
        W, bq = models.general_hmpo(ch, (2,), H, ops, [(f"X{i}", f"X{i}", jp) for i in range(4)])
        return ch, W, bq
    ch, W0, bq = mpo(g0, jp0)
    if which == "g":
        dW = 0.5 * (mpo(g0 + 1.0, jp0)[1] - mpo(g0 - 1.0, jp0)[1])
        Wp, Wm = mpo(g0 + h, jp0)[1], mpo(g0 - h, jp0)[1]
    else:
        dW = 0.5 * (mpo(g0, jp0 + 1.0)[1] - mpo(g0, jp0 - 1.0)[1])
        Wp, Wm = mpo(g0, jp0 + h)[1], mpo(g0, jp0 - h)[1]
    T = lambda W: models.mpo_tensor(ch, W, bq)
    run = iDMRG(ctx, (2,), T(W0), tol=1e-13, krylov_dim=32, gradient=T(dW))
    rp = iDMRG(ctx, (2,), T(Wp), tol=1e-13, krylov_dim=32)
    rm = iDMRG(ctx, (2,), T(Wm), tol=1e-13, krylov_dim=32)
    for step in range(2):
        a = run.grow(128, 0.0)
        fd = (rp.grow(128, 0.0)["energy"] - rm.grow(128, 0.0)["energy"]) / (2 * h)
        assert a["truncation"] == 0.0
        assert abs(a["gradient"] - fd) <= 1e-6 * max(1.0, abs(fd)), (which, step, a["gradient"], fd)


def test_fdmrg_gradient_through_sweeps(ctx):
    """dE/dJz carried through finite DMRG: growth to 10 vertices and two
    sweeps at chi = 64 (no truncation: bond dimensions up to 32), the
    derivative blocks updated with every sweep step's factors.  Every
    energies-file row's gradient against central differences (h = 1e-4) of
    the same row's energy, to 1e-6 relative; the mixed-precision run within
    1e-8 of the FP64 one."""
    from chainamps_b200 import fDMRG, models, CMPS_SPLIT_TF32
    jz, h = 0.7, 1e-4
    rules, ch, W0, bq = xxz_mpo(jz)
    dW = 0.5 * (xxz_mpo(jz + 1.0)[2] - xxz_mpo(jz - 1.0)[2])
    T = lambda W: models.mpo_tensor(ch, W, bq)
    rows = fDMRG(ctx, rules, T(W0), 10, tol=1e-13, krylov_dim=32, gradient=T(dW)).run(2, 64, 0.0)
    mixed = fDMRG(ctx, rules, T(W0), 10, precision=CMPS_SPLIT_TF32, tol=1e-13, krylov_dim=32,
                  gradient=T(dW)).run(2, 64, 0.0)
    rp = fDMRG(ctx, rules, T(xxz_mpo(jz + h)[2]), 10, tol=1e-13, krylov_dim=32).run(2, 64, 0.0)
    rm = fDMRG(ctx, rules, T(xxz_mpo(jz - h)[2]), 10, tol=1e-13, krylov_dim=32).run(2, 64, 0.0)
    assert len(rows) == len(rp) == len(rm) == len(mixed) > 5
    for a, b, p, m in zip(rows, mixed, rp, rm):
        assert a["truncation"] == 0.0
        fd = (p["energy"] - m["energy"]) / (2 * h)
        assert abs(a["gradient"] - fd) <= 1e-6 * max(1.0, abs(fd)), (a, fd)
        assert abs(b["gradient"] - a["gradient"]) <= 1e-8 * max(1.0, abs(a["gradient"])), (b, a)
