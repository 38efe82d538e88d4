"""The PaScaL_TDMA heat example, restated on one rank as a caller of the
PaScaL_TDMA interface (test infrastructure, imported by the tests only).

The reference ships this example beside the library (PaScaL_TDMA/examples):
three-dimensional heat conduction in a unit cube, walls at y = 0 (hot) and
y = ly (cold), periodic in x and z, advanced by an approximately factored
Crank-Nicolson step whose three sweeps are PaScaL_TDMA many-system solves
(solve_theta_plan_many.f90) or one single-system solve per line
(solve_theta_plan_single.f90).  The restatement keeps:
  * the parameters of global.f90:91-107 (Pr = 5, Ra = 200, dt = 5e-3,
    theta_hot = 1, theta_cold = -1, nu = 1/sqrt(Ra/(Pr ly^3 dT)), Ct = nu/Pr);
  * the one-rank mesh of mpi_subdomain.f90:272-329 (x, z vertex-periodic,
    y with walls at j = 0 and j = ny_sub, dmy_sub(0) = dy/2);
  * the initial field of :339-364 and the wall arrays of :372-405;
  * the y-boundary flags of :255-268;
  * the ghost update of :222-248 (periodic x and z; y has no neighbour);
  * the right-hand side, the coefficient rows and the sweep order of
    solve_theta_plan_many.f90:59-216 and solve_theta_plan_single.f90,
    expression by expression, with a plan created and destroyed around
    every sweep as the example does.

The solver is pluggable, so the same driver runs on the GPU library and on
the oracle.  Because the field starts as the linear conduction profile plus
one separable sine mode that the discrete operators have as an eigenvector,
every step multiplies the mode by a closed-form factor (`mode_factor`): a
known answer for the whole example that depends on neither implementation.
"""
import math

import numpy as np


class HeatExample:
    """State of the example on one rank.  theta is stored [k, j, i] (i fastest,
    the Fortran theta_sub(0:nx_sub, 0:ny_sub, 0:nz_sub) memory order)."""

    def __init__(self, nx: int, ny: int, nz: int):
        # PARA_INPUT meshes (global.f90:91-96 add one to each)
        self.NX, self.NY, self.NZ = nx + 1, ny + 1, nz + 1
        # para_range(1, n-1) on one rank: ista = 1, iend = n-1, n_sub = n
        NX, NY, NZ = self.NX, self.NY, self.NZ
        self.Pr, self.Ra = 5.0, 2.0e2
        self.dt = 5.0e-3
        self.lx = self.ly = self.lz = 1.0
        self.theta_cold = -1.0
        self.theta_hot = 2.0 + self.theta_cold
        alphaG = 1.0
        self.nu = 1.0 / math.sqrt(self.Ra / (alphaG * self.Pr * self.ly ** 3.0 * (self.theta_hot - self.theta_cold)))
        self.Ct = self.nu / self.Pr
        # mesh (mpi_subdomain_mesh): one rank holds rank 0 of every direction,
        # so only the rank-0 branches apply (dmy_sub(ny_sub) stays dy)
        self.dx = self.lx / (NX - 1)
        self.dy = self.ly / NY
        self.dz = self.lz / (NZ - 1)
        self.X = (np.arange(NX + 1) - 1) * self.dx
        self.Y = np.arange(NY + 1) * self.dy
        self.Z = (np.arange(NZ + 1) - 1) * self.dz
        self.Y[0] = 0.0
        self.dmx = np.full(NX + 1, self.dx)
        self.dmy = np.full(NY + 1, self.dy)
        self.dmy[0] = self.dy / 2.0
        self.dmz = np.full(NZ + 1, self.dz)
        # mpi_subdomain_indices: the first and last interior rows see a wall
        self.jmbc = np.ones(NY + 1, dtype=np.int64)
        self.jpbc = np.ones(NY + 1, dtype=np.int64)
        self.jmbc[1] = 0
        self.jpbc[NY - 1] = 0
        # mpi_subdomain_initialization
        pi = math.pi
        base = (self.theta_cold - self.theta_hot) / self.ly * self.Y + self.theta_hot
        sx = np.sin(2 * 2.0 * pi / self.lx * self.X)
        sz = np.sin(2 * 2.0 * pi / self.lz * self.Z)
        sy = np.sin(2 * 2.0 * pi / self.ly * self.Y)
        th = base[None, :, None] + sx[None, None, :] * sz[:, None, None] * sy[None, :, None]
        th[:, 0, :] = self.theta_hot
        th[:, NY, :] = self.theta_cold
        self.theta = np.ascontiguousarray(th)
        self.ghost_update()
        # mpi_subdomain_boundary (rank 0 of y): [k, i]
        self.BC3 = np.full((NZ + 1, NX + 1), self.theta_hot)
        self.BC4 = self.theta[:, NY, :].copy()
        # the parts of the initial field the closed form follows
        self.base0 = base.copy()
        self.mode0 = (sx[None, None, :] * sz[:, None, None] * sy[None, :, None])

    def ghost_update(self) -> None:
        """Periodic faces in x then z (mpi_subdomain.f90:222-248 on one rank;
        the x and z exchanges touch different cells except the edges, which
        no stencil reads)."""
        t, NX, NZ = self.theta, self.NX, self.NZ
        t[:, :, 0] = t[:, :, NX - 1]
        t[:, :, NX] = t[:, :, 1]
        t[0, :, :] = t[NZ - 1, :, :]
        t[NZ, :, :] = t[1, :, :]

    def rhs(self) -> np.ndarray:
        """solve_theta_plan_many.f90:59-127: the explicit right-hand side on
        the interior, [k, j, i]."""
        T, Ct, dt = self.theta, self.Ct, self.dt
        dx, dy, dz = self.dx, self.dy, self.dz
        c = T[1:-1, 1:-1, 1:-1]
        Txm, Txp = T[1:-1, 1:-1, :-2], T[1:-1, 1:-1, 2:]
        Tym, Typ = T[1:-1, :-2, 1:-1], T[1:-1, 2:, 1:-1]
        Tzm, Tzp = T[:-2, 1:-1, 1:-1], T[2:, 1:-1, 1:-1]
        dmx_i, dmx_ip = self.dmx[1:-1][None, None, :], self.dmx[2:][None, None, :]
        dmy_j, dmy_jp = self.dmy[1:-1][None, :, None], self.dmy[2:][None, :, None]
        dmz_k, dmz_kp = self.dmz[1:-1][:, None, None], self.dmz[2:][:, None, None]
        jem = self.jmbc[1:-1][None, :, None].astype(np.float64)
        jep = self.jpbc[1:-1][None, :, None].astype(np.float64)
        dedx1 = (c - Txm) / dmx_i
        dedx2 = (Txp - c) / dmx_ip
        dedy3 = (c - Tym) / dmy_j
        dedy4 = (Typ - c) / dmy_jp
        dedz5 = (c - Tzm) / dmz_k
        dedz6 = (Tzp - c) / dmz_kp
        e1 = 1.0 / dx * (dedx2 - dedx1)
        e2 = 1.0 / dy * (dedy4 - dedy3)
        e3 = 1.0 / dz * (dedz6 - dedz5)
        viscous = 0.5 * Ct * (e1 + e2 + e3)
        ebc_down = 0.5 * Ct / dy / dmy_j * self.BC3[1:-1, None, 1:-1]
        ebc_up = 0.5 * Ct / dy / dmy_jp * self.BC4[1:-1, None, 1:-1]
        ebc = (1.0 - jem) * ebc_down + (1.0 - jep) * ebc_up
        eAPI = -(0.5 * Ct / dx / dmx_ip)
        eAMI = -(0.5 * Ct / dx / dmx_i)
        eACI = 0.5 * Ct / dx * (1.0 / dmx_ip + 1.0 / dmx_i)
        eAPK = -(0.5 * Ct / dz / dmz_kp)
        eAMK = -(0.5 * Ct / dz / dmz_k)
        eACK = 0.5 * Ct / dz * (1.0 / dmz_kp + 1.0 / dmz_k)
        eAPJ = -(0.5 * Ct / dy * (1.0 / dmy_jp) * jep)
        eAMJ = -(0.5 * Ct / dy * (1.0 / dmy_j) * jem)
        eACJ = 0.5 * Ct / dy * (1.0 / dmy_jp + 1.0 / dmy_j)
        eRHS = (eAPK * Tzp + eACK * c + eAMK * Tzm
                + eAPJ * Typ + eACJ * c + eAMJ * Tym
                + eAPI * Txp + eACI * c + eAMI * Txm)
        return np.ascontiguousarray(c / dt + viscous + ebc - (c / dt + eRHS))

    # coefficient rows of the three sweeps, as the example builds them
    def _rows_z(self):
        Ct, dt, dz = self.Ct, self.dt, self.dz
        dmz_k, dmz_kp = self.dmz[1:-1], self.dmz[2:]
        ap = -(0.5 * Ct / dz / dmz_kp * dt)
        am = -(0.5 * Ct / dz / dmz_k * dt)
        ac = 0.5 * Ct / dz * (1.0 / dmz_kp + 1.0 / dmz_k) * dt + 1.0
        return am, ac, ap

    def _rows_y(self):
        Ct, dt, dy = self.Ct, self.dt, self.dy
        dmy_j, dmy_jp = self.dmy[1:-1], self.dmy[2:]
        jem = self.jmbc[1:-1].astype(np.float64)
        jep = self.jpbc[1:-1].astype(np.float64)
        ap = -(0.5 * Ct / dy / dmy_jp * jep * dt)
        am = -(0.5 * Ct / dy / dmy_j * jem * dt)
        ac = 0.5 * Ct / dy * (1.0 / dmy_jp + 1.0 / dmy_j) * dt + 1.0
        return am, ac, ap

    def _rows_x(self):
        Ct, dt, dx = self.Ct, self.dt, self.dx
        dmx_i, dmx_ip = self.dmx[1:-1], self.dmx[2:]
        ap = -(0.5 * Ct / dx / dmx_ip * dt)
        am = -(0.5 * Ct / dx / dmx_i * dt)
        ac = 0.5 * Ct / dx * (1.0 / dmx_ip + 1.0 / dmx_i) * dt + 1.0
        return am, ac, ap

    def step_many(self, make_plan, nonblocking: bool = False) -> None:
        """solve_theta_plan_many.f90: z sweep (cyclic, one (x, z) plane of
        lines per j), the y sweep (one (x, y) plane per k) and the x sweep
        (cyclic, one (y, x) plane per k), each through a plan of its own.
        make_plan(n_sys) returns an object with many_solve, many_solve_cycle
        (and their _nonblocking forms) and destroy."""
        NX, NY, NZ = self.NX, self.NY, self.NZ
        sfx = "_nonblocking" if nonblocking else ""
        rhs = self.rhs()
        # z: ap(1:nx_sub-1, 1:nz_sub-1), system index i fastest -> [k, i]
        am1, ac1, ap1 = self._rows_z()
        plan = make_plan(NX - 1)
        for j in range(NY - 1):
            am = np.ascontiguousarray(np.broadcast_to(am1[:, None], (NZ - 1, NX - 1)))
            ac = np.ascontiguousarray(np.broadcast_to(ac1[:, None], (NZ - 1, NX - 1)))
            ap = np.ascontiguousarray(np.broadcast_to(ap1[:, None], (NZ - 1, NX - 1)))
            ad = np.ascontiguousarray(rhs[:, j, :] * self.dt)
            getattr(plan, "many_solve_cycle" + sfx)(am, ac, ap, ad, NX - 1, NZ - 1)
            rhs[:, j, :] = ad
        plan.destroy()
        # y: ap(1:nx_sub-1, 1:ny_sub-1) -> [j, i]
        am1, ac1, ap1 = self._rows_y()
        plan = make_plan(NX - 1)
        for k in range(NZ - 1):
            am = np.ascontiguousarray(np.broadcast_to(am1[:, None], (NY - 1, NX - 1)))
            ac = np.ascontiguousarray(np.broadcast_to(ac1[:, None], (NY - 1, NX - 1)))
            ap = np.ascontiguousarray(np.broadcast_to(ap1[:, None], (NY - 1, NX - 1)))
            ad = np.ascontiguousarray(rhs[k, :, :])
            getattr(plan, "many_solve" + sfx)(am, ac, ap, ad, NX - 1, NY - 1)
            rhs[k, :, :] = ad
        plan.destroy()
        # x: ap(1:ny_sub-1, 1:nx_sub-1), system index j fastest -> [i, j]
        am1, ac1, ap1 = self._rows_x()
        plan = make_plan(NY - 1)
        for k in range(NZ - 1):
            am = np.ascontiguousarray(np.broadcast_to(am1[:, None], (NX - 1, NY - 1)))
            ac = np.ascontiguousarray(np.broadcast_to(ac1[:, None], (NX - 1, NY - 1)))
            ap = np.ascontiguousarray(np.broadcast_to(ap1[:, None], (NX - 1, NY - 1)))
            ad = np.ascontiguousarray(rhs[k, :, :].T)
            getattr(plan, "many_solve_cycle" + sfx)(am, ac, ap, ad, NY - 1, NX - 1)
            self.theta[k + 1, 1:-1, 1:-1] = self.theta[k + 1, 1:-1, 1:-1] + ad.T
        plan.destroy()
        self.ghost_update()

    def step_single(self, make_plan) -> None:
        """solve_theta_plan_single.f90: the same three sweeps, one
        single-system solve per line.  make_plan() returns an object with
        single_solve, single_solve_cycle and destroy."""
        NX, NY, NZ = self.NX, self.NY, self.NZ
        rhs = self.rhs()
        am1, ac1, ap1 = self._rows_z()
        plan = make_plan()
        for j in range(NY - 1):
            for i in range(NX - 1):
                am, ac, ap = am1.copy(), ac1.copy(), ap1.copy()
                ad = np.ascontiguousarray(rhs[:, j, i] * self.dt)
                plan.single_solve_cycle(am, ac, ap, ad, NZ - 1)
                rhs[:, j, i] = ad
        plan.destroy()
        am1, ac1, ap1 = self._rows_y()
        plan = make_plan()
        for k in range(NZ - 1):
            for i in range(NX - 1):
                am, ac, ap = am1.copy(), ac1.copy(), ap1.copy()
                ad = np.ascontiguousarray(rhs[k, :, i])
                plan.single_solve(am, ac, ap, ad, NY - 1)
                rhs[k, :, i] = ad
        plan.destroy()
        am1, ac1, ap1 = self._rows_x()
        plan = make_plan()
        for k in range(NZ - 1):
            for j in range(NY - 1):
                am, ac, ap = am1.copy(), ac1.copy(), ap1.copy()
                ad = np.ascontiguousarray(rhs[k, j, :])
                plan.single_solve_cycle(am, ac, ap, ad, NX - 1)
                self.theta[k + 1, j + 1, 1:-1] = self.theta[k + 1, j + 1, 1:-1] + ad
        plan.destroy()
        self.ghost_update()

    def mode_factor(self) -> float:
        """The factor one step multiplies the sine mode by.  With L the
        discrete Laplacian, the right-hand side is Ct L theta (the wall terms
        of the explicit and implicit parts cancel against ebc), the linear
        profile has L theta0 = 0, and sin(4 pi x/lx) sin(4 pi y/ly)
        sin(4 pi z/lz) is an eigenvector of each one-dimensional operator
        (periodic in x and z, Dirichlet at the walls in y) with eigenvalue
        -4 sin^2(k h/2)/h^2.  So the step is
            theta' - theta0 = (1 + dt Ct S / prod_d (1 - dt Ct lam_d / 2)) (theta - theta0),
        S = lam_x + lam_y + lam_z."""
        k = 4.0 * math.pi
        lam = [-4.0 * math.sin(k / L * h / 2.0) ** 2 / h ** 2
               for L, h in ((self.lx, self.dx), (self.ly, self.dy), (self.lz, self.dz))]
        a = self.dt * self.Ct
        den = 1.0
        for l in lam:
            den *= 1.0 - 0.5 * a * l
        return 1.0 + a * sum(lam) / den

    def expected(self, nsteps: int) -> np.ndarray:
        """The interior field after nsteps, from the closed form."""
        g = self.mode_factor() ** nsteps
        want = self.base0[None, :, None] + g * self.mode0
        return want[1:-1, 1:-1, 1:-1]

    def interior(self) -> np.ndarray:
        return self.theta[1:-1, 1:-1, 1:-1].copy()


class OraclePlan:
    """A PaScaL_TDMA plan over the oracle's one-rank solves (the test
    oracle's tdma_many restates pascal_tdma.f90:487-578 and 715-806; the
    single-system solves do the same arithmetic with one system,
    tdmas.f90:27-100)."""

    def __init__(self, oracle_mod, n_sys: int = 1):
        self.O, self.n_sys = oracle_mod, n_sys

    def _many(self, A, B, C, D, n_sys, n_row, cyclic):
        assert n_sys == self.n_sys and D.shape == (n_row, n_sys)
        D[...] = self.O.tdma_many(A, B, C, D, cyclic=cyclic)

    def many_solve(self, A, B, C, D, n_sys, n_row):
        self._many(A, B, C, D, n_sys, n_row, False)

    def many_solve_cycle(self, A, B, C, D, n_sys, n_row):
        self._many(A, B, C, D, n_sys, n_row, True)

    many_solve_nonblocking = many_solve
    many_solve_cycle_nonblocking = many_solve_cycle

    def single_solve(self, A, B, C, D, n_row):
        D[...] = self.O.tdma_many(A[:, None], B[:, None], C[:, None], D[:, None], cyclic=False)[:, 0]

    def single_solve_cycle(self, A, B, C, D, n_row):
        D[...] = self.O.tdma_many(A[:, None], B[:, None], C[:, None], D[:, None], cyclic=True)[:, 0]

    def destroy(self):
        pass
