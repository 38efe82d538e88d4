"""Known-answer tests that pin the CPU oracle (no GPU needed).

The reference ships no golden vectors and cannot be built here (Fortran 90 +
MPI + FFTW), so the oracle is pinned component by component against
mathematics: dense solves for PaScaL_TDMA (pascal_tdma.f90:487-806), an
O(n^2) DFT for the FFTW stand-in, the discrete Poisson operator that
mpi_pressure_Poisson_FFT2 inverts (module_solve_pressure.f90:489-744), and the
post-projection divergence invariant that main.f90:205-212 monitors.
"""
import numpy as np
import pytest

RTOL = 1e-12


def _dominant(rng, n_row, n_sys, ratio=0.3):
    A = rng.uniform(-1, 1, (n_row, n_sys)) * ratio
    C = rng.uniform(-1, 1, (n_row, n_sys)) * ratio
    B = 1.0 + rng.uniform(0, 1, (n_row, n_sys))
    D = rng.uniform(-1, 1, (n_row, n_sys))
    return A, B, C, D


def _dense(A, B, C, s, cyclic):
    n = A.shape[0]
    M = np.zeros((n, n))
    for r in range(n):
        M[r, r] = B[r, s]
        if r > 0:
            M[r, r - 1] = A[r, s]
        elif cyclic:
            M[r, n - 1] += A[r, s]
        if r < n - 1:
            M[r, r + 1] = C[r, s]
        elif cyclic:
            M[r, 0] += C[r, s]
    return M


@pytest.mark.parametrize("n_row", [3, 4, 7, 64, 129])
def test_tdma_many_matches_dense(oracle_mod, n_row):
    rng = np.random.default_rng(n_row)
    A, B, C, D = _dominant(rng, n_row, 9)
    X = oracle_mod.tdma_many(A, B, C, D, cyclic=False)
    for s in range(9):
        ref = np.linalg.solve(_dense(A, B, C, s, cyclic=False), D[:, s])
        np.testing.assert_allclose(X[:, s], ref, rtol=RTOL, atol=1e-14)


@pytest.mark.parametrize("n_row", [3, 5, 16, 64, 96])
def test_tdma_many_cycle_matches_dense(oracle_mod, n_row):
    # |a/b| <= 0.15: the dropped closure coefficient is O(0.15^(n-1)), invisible.
    rng = np.random.default_rng(100 + n_row)
    A, B, C, D = _dominant(rng, n_row, 7, ratio=0.15)
    X = oracle_mod.tdma_many(A, B, C, D, cyclic=True)
    for s in range(7):
        ref = np.linalg.solve(_dense(A, B, C, s, cyclic=True), D[:, s])
        tol = 1e-12 if n_row >= 16 else 0.15 ** (n_row - 1) * 10
        np.testing.assert_allclose(X[:, s], ref, rtol=tol, atol=tol)


def _modified_thomas_py(a, b, c, d, cyclic):
    """Independent scalar restatement of pascal_tdma.f90:487-578 / 715-806 with
    the one-rank reduced solve of tdmas.f90:113-146 / 159-212."""
    a, b, c, d = (list(map(float, v)) for v in (a, b, c, d))
    n = len(d)
    for r in (0, 1):
        a[r] /= b[r]; d[r] /= b[r]; c[r] /= b[r]
    for j in range(2, n):
        r = 1.0 / (b[j] - a[j] * c[j - 1])
        d[j] = r * (d[j] - a[j] * d[j - 1])
        c[j] = r * c[j]
        a[j] = -r * a[j] * a[j - 1]
    for j in range(n - 3, 0, -1):
        d[j] = d[j] - c[j] * d[j + 1]
        a[j] = a[j] - c[j] * a[j + 1]
        c[j] = -c[j] * c[j + 1]
    r = 1.0 / (1.0 - a[1] * c[0])
    d[0] = r * (d[0] - c[0] * d[1])
    a[0] = r * a[0]
    c[0] = -r * c[0] * c[1]
    a1, c1, d1, a2, c2, d2 = a[0], c[0], d[0], a[n - 1], c[n - 1], d[n - 1]
    if cyclic:
        e2 = -c2                       # e(2) = -a(2) is overwritten by e(n2) = -c(n2)
        x1 = (d1 - a1 * d2 - c1 * d2) / (1.0 + a1 * e2 + c1 * e2)
        x2 = d2 + x1 * e2
    else:
        r = 1.0 / (1.0 - a2 * c1)
        x2 = r * (d2 - a2 * d1)
        x1 = d1 - c1 * x2
    d[0], d[n - 1] = x1, x2
    for j in range(1, n - 1):
        d[j] = d[j] - a[j] * d[0] - c[j] * d[n - 1]
    return np.array(d)


@pytest.mark.parametrize("cyclic", [False, True])
def test_tdma_restatement_bitwise_incl_cyclic_closure(oracle_mod, cyclic):
    # Weakly dominant systems where the one-rank cyclic closure (A_rd(:,2)
    # dropped) is visible: the C oracle must agree bit for bit with an
    # independent scalar restatement of the same arithmetic.
    rng = np.random.default_rng(7)
    n_row, n_sys = 6, 5
    A, B, C, D = _dominant(rng, n_row, n_sys, ratio=0.45)
    X = oracle_mod.tdma_many(A, B, C, D, cyclic=cyclic)
    for s in range(n_sys):
        ref = _modified_thomas_py(A[:, s], B[:, s], C[:, s], D[:, s], cyclic)
        assert np.array_equal(X[:, s], ref)
    if cyclic:  # and the closure really differs from the exact cyclic solve here
        ex = np.linalg.solve(_dense(A, B, C, 0, cyclic=True), D[:, 0])
        assert np.max(np.abs(X[:, 0] - ex)) > 1e-9


def test_tdma_noncyclic_ignores_outer_couplings(oracle_mod):
    rng = np.random.default_rng(3)
    A, B, C, D = _dominant(rng, 10, 4)
    X1 = oracle_mod.tdma_many(A, B, C, D)
    A[0, :] = 123.0
    C[-1, :] = -77.0
    X2 = oracle_mod.tdma_many(A, B, C, D)
    np.testing.assert_array_equal(X1, X2)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 8, 12, 30, 60, 64, 96, 160, 192])
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft_matches_direct_dft(oracle_mod, n, sign):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((3, n)) + 1j * rng.standard_normal((3, n))
    k = np.arange(n)
    Wm = np.exp(sign * 2j * np.pi * np.outer(k, k) / n)
    ref = x @ Wm.T
    got = oracle_mod.fft_c2c(x, sign)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-12 * max(1, n))
    npref = np.fft.fft(x, axis=-1) if sign < 0 else np.fft.ifft(x, axis=-1) * n
    np.testing.assert_allclose(got, npref, rtol=1e-13, atol=1e-12 * max(1, n))


def _discrete_laplacian(o, dP):
    """The operator inverted by mpi_pressure_Poisson_FFT2: periodic 3-point
    second differences in x and z on the uniform spacing L/n (the modified
    wavenumbers of :93-129) and the y stencil of :599-626 with zero flux at the
    walls.  dP is (n3m, n2m, n1m)."""
    p = o.params
    L1 = p["H"] * p["aspect1"]; L3 = p["H"] * p["aspect3"]
    ddx = L1 / p["n1m"]; ddz = L3 / p["n3m"]
    dx2 = o.metric("dx2"); dmx2 = o.metric("dmx2")
    n2 = p["n2m"]
    lap = (np.roll(dP, -1, 2) - 2 * dP + np.roll(dP, 1, 2)) / (ddx * ddx)
    lap += (np.roll(dP, -1, 0) - 2 * dP + np.roll(dP, 1, 0)) / (ddz * ddz)
    for j in range(1, n2 + 1):
        am = 0.0 if j == 1 else 1.0 / dx2[j] / dmx2[j]
        ap = 0.0 if j == n2 else 1.0 / dx2[j] / dmx2[j + 1]
        y = -(am + ap) * dP[:, j - 1, :]
        if j > 1:
            y += am * dP[:, j - 2, :]
        if j < n2:
            y += ap * dP[:, j, :]
        lap[:, j - 1, :] += y
    return lap


@pytest.mark.parametrize("dims", [(16, 12, 10), (32, 24, 20), (30, 16, 18)])
def test_poisson_inverts_discrete_operator(oracle_mod, dims):
    n1, n2, n3 = dims
    o = oracle_mod.Oracle(n1m=n1, n2m=n2, n3m=n3)
    rng = np.random.default_rng(sum(dims))
    dP = rng.standard_normal((n3, n2, n1))
    o.set_prhs(_discrete_laplacian(o, dP))
    o.stage("poisson")
    got = o.get("dP")[1:-1, 1:-1, 1:-1]
    np.testing.assert_allclose(got, dP - dP.mean(), rtol=0, atol=1e-10 * np.abs(dP).max())


def test_poisson_ghosts_and_wall_extrapolation(oracle_mod):
    o = oracle_mod.Oracle(n1m=16, n2m=12, n3m=10)
    rng = np.random.default_rng(5)
    o.set_prhs(rng.standard_normal((10, 12, 16)))
    o.stage("poisson")
    dP = o.get("dP")
    np.testing.assert_array_equal(dP[:, :, 0], dP[:, :, -2])     # x ghosts
    np.testing.assert_array_equal(dP[:, :, -1], dP[:, :, 1])
    np.testing.assert_array_equal(dP[0], dP[-2])                 # z ghosts (after x)
    np.testing.assert_array_equal(dP[-1], dP[1])
    dmx2 = o.metric("dmx2")
    a = (dmx2[1] + dmx2[2]) ** 2 / ((dmx2[1] + dmx2[2]) ** 2 - dmx2[1] ** 2)
    b = dmx2[1] ** 2 / ((dmx2[1] + dmx2[2]) ** 2 - dmx2[1] ** 2)
    np.testing.assert_allclose(dP[1:-1, 0, 1:-1], a * dP[1:-1, 1, 1:-1] - b * dP[1:-1, 2, 1:-1], rtol=1e-14)


def test_mesh_matches_reference_formulas(oracle_mod):
    o = oracle_mod.Oracle(n1m=16, n2m=12, n3m=10, gamma2=1.5)
    x1, dx1, dmx1 = o.metric("x1"), o.metric("dx1"), o.metric("dmx1")
    i = np.arange(18)
    np.testing.assert_array_equal(x1, (i - 1) * 2.0 / 16)
    assert dx1[0] == dx1[16] and dx1[17] == dx1[1] and dmx1[0] == dmx1[16]
    x2, dx2, dmx2 = o.metric("x2"), o.metric("dx2"), o.metric("dmx2")
    j = np.arange(1, 14)
    ref = 0.5 * (1 + np.tanh(0.5 * 1.5 * (2.0 * (j - 1) / 12 - 1.0)) / np.tanh(1.5 * 0.5))
    np.testing.assert_allclose(x2[1:], ref, rtol=1e-15, atol=1e-16)
    assert x2[0] == x2[1] and dx2[0] == 0 and dx2[13] == 0
    assert dmx2[1] == 0.5 * dx2[1] and dmx2[13] == 0.5 * dx2[12]
    np.testing.assert_allclose(dx2[1:13].sum(), 1.0, rtol=1e-14)


def test_step_is_divergence_free_and_finite(oracle_mod):
    o = oracle_mod.Oracle(n1m=24, n2m=20, n3m=16)
    d = o.step(8)
    assert np.all(np.isfinite(d))
    assert np.all(np.abs(d[:, 2]) < 1e-12)       # signed max divergence after projection
    T = o.get("T")
    assert np.all(T[1:-1, 0, 1:-1] == 0.5)        # bottom wall ghost row
    assert np.all(T[1:-1, -1, 1:-1] == 0.0)       # one-rank top ghost row stays 0


def test_initial_field_is_seeded_conduction_profile(oracle_mod):
    o = oracle_mod.Oracle(n1m=16, n2m=12, n3m=10, seed=3)
    T = o.get("T")[1:-1, 1:-1, 1:-1]
    x2 = o.metric("x2")
    yc = 0.5 * (x2[1:13] + x2[2:14])
    dev = T - (0.5 - yc)[None, :, None]
    assert np.all(np.abs(dev) <= 0.01) and abs(dev.mean()) < 2e-3 and dev.std() > 4e-3
    o2 = oracle_mod.Oracle(n1m=16, n2m=12, n3m=10, seed=3)
    np.testing.assert_array_equal(o2.get("T"), o.get("T"))
    o3 = oracle_mod.Oracle(n1m=16, n2m=12, n3m=10, seed=4)
    assert not np.array_equal(o3.get("T"), o.get("T"))


def test_row_wise_momentum_coefficients(oracle_mod):
    # mpi_momentum_coeffi assigns Mu(:,j,k) inside the i loop: every row holds f(T(n1sub,j,k)).
    o = oracle_mod.Oracle(n1m=16, n2m=12, n3m=10, property_set=1, Pr=7.0)
    o.stage("thermal"); o.stage("ghost_T"); o.stage("mom_coeffi")
    Mu = o.get("Mu")
    assert np.all(Mu == Mu[:, :, -1:])
    assert np.ptp(Mu[1:-1, 1:-1, 1]) > 0
