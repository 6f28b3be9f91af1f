"""The study's larger domain-wall configurations on the GPU, at full size.

* Nt = 64 with Nx in {32, 56, 80, 96}, Ls = 16, m_f = 0.05, beta = 3 (the
  analyzer's finite-volume scan): propagators by the even-odd mixed solver and
  by the plain FP64 CG agree, meet the FP64 true residual of the normal
  equation independently recomputed by the CPU oracle, and the analyzer's
  correlators from both solvers agree.
* 128x128, Ls = 24, M5 = 1, m_f = 0.02, beta = 4 (the large HMC run): one
  trajectory with the FP64 CG and with the mixed CG from identical draws
  gives the same proposal, dH and plaquette; propagators as above.

The CPU oracle is too slow for whole solves at these sizes, so parity here
rests on size-independent checks: the oracle's own operator applied to the
GPU solutions, and agreement between solvers that share no kernels."""
import numpy as np
import pytest

from conftest import quenched_theta, random_field, rel
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T():
    import three_part_dwf_study_b200 as T
    return T


def analyzer_sources(rng, Nt, Nx, Ls):
    """Two boundary point sources (spin 1 on s = 0, spin 0 on s = Ls-1), two
    boundary Z4 noise sources and one boundary wall source."""
    n = Ls * Nt * Nx * 2
    srcs = []
    for t, b in ((0, 1), (Nt // 2, 0)):
        v = np.zeros((Ls, Nt, Nx, 2), np.complex128)
        v[0 if b == 1 else Ls - 1, t, 0, b] = 1.0
        srcs.append(v.ravel())
    for _ in range(2):
        eta = np.exp(0.5j * np.pi * rng.integers(0, 4, size=(Nt, Nx, 2)))
        v = np.zeros((Ls, Nt, Nx, 2), np.complex128)
        v[0, :, :, 1] = eta[:, :, 1]
        v[Ls - 1, :, :, 0] = eta[:, :, 0]
        srcs.append(v.ravel())
    v = np.zeros((Ls, Nt, Nx, 2), np.complex128)
    v[0, Nt // 4, :, 1] = 1.0
    srcs.append(v.ravel())
    out = np.stack(srcs)
    assert out.shape[1] == n
    return out


def check_propagators(T, d, o, th, src):
    x_eo, info_eo = d.propagators(src, rtol=1e-10, maxiter=50000, solver=T.SOLVER_EO_MIXED)
    x_64, info_64 = d.propagators(src, rtol=1e-10, maxiter=50000, solver=T.SOLVER_CG64)
    for k in range(src.shape[0]):
        assert info_eo[k]["converged"] and info_64[k]["converged"]
        assert info_eo[k]["schur_iterations"] > 0
        # the reference's stopping rule recomputed by the oracle's operator:
        # |D^dag D x - D^dag src| / |D^dag src| <= 1e-10
        rhs = o.apply(1, th, src[k])
        for x in (x_eo[k], x_64[k]):
            r = o.apply(3, th, x) - rhs
            assert np.linalg.norm(r) / np.linalg.norm(rhs) <= 1.0e-10 * 1.001
        assert rel(x_eo[k], x_64[k]) < 1e-7


@pytest.mark.parametrize("Nx", [32, 56, 80, 96])
def test_finite_volume_scan_propagators_and_correlators(T, Nx):
    from three_part_dwf_study_b200.rng import z4_digits
    Nt, Ls, mf, beta = 64, 16, 0.05, 3.0
    rng = np.random.default_rng(500 + Nx)
    th = quenched_theta(rng, Nt, Nx, beta)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, mf, beta)
    o = O.Dwf(Nt, Nx, Ls, 1.0, mf)
    d.set_gauge(th)
    check_propagators(T, d, o, th, analyzer_sources(rng, Nt, Nx, Ls))
    z4 = z4_digits(918273, 2 * Nt * Nx * 2)
    ms = [d.measure(th, z4=z4, n_point_times=2, n_wall_times=2, n_noise=2, max_momentum=3,
                    rtol=1e-10, maxiter=50000, solver=sv)
          for sv in (T.SOLVER_EO_MIXED, T.SOLVER_CG64)]
    for key in ("cpp", "cj5", "mom_cpp", "loop"):
        assert rel(ms[0][key], ms[1][key]) < 1e-7, key
    assert all(i["converged"] for m in ms for i in m["info"])
    d.close()


def test_large_lattice_propagators(T):
    Nt, Nx, Ls, mf, beta = 128, 128, 24, 0.02, 4.0
    rng = np.random.default_rng(128)
    th = quenched_theta(rng, Nt, Nx, beta)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, mf, beta)
    o = O.Dwf(Nt, Nx, Ls, 1.0, mf)
    d.set_gauge(th)
    check_propagators(T, d, o, th, analyzer_sources(rng, Nt, Nx, Ls)[[0, 2]])
    d.close()


def test_large_lattice_hmc_fp64_and_mixed_agree(T):
    Nt, Nx, Ls, mf, beta = 128, 128, 24, 0.02, 4.0
    eps, steps = 0.02, 5
    rng = np.random.default_rng(4)
    th0 = quenched_theta(rng, Nt, Nx, beta)
    d = T.DomainWall(Nt, Nx, Ls, 1.0, mf, beta)
    chi = random_field(rng, d.Ndof)
    mom = rng.normal(size=d.Ngauge)
    res = {}
    for sv in (T.SOLVER_CG64, T.SOLVER_MIXED):
        res[sv] = d.hmc_trajectory(th0, chi, mom, eps, steps, rtol=1e-10, maxiter=50000, solver=sv)
    (o64, i64), (omx, imx) = res[T.SOLVER_CG64], res[T.SOLVER_MIXED]
    assert i64["solves"] == imx["solves"] == steps + 1
    assert abs(i64["dH"] - imx["dH"]) < 1e-6
    assert abs(i64["H0"] - imx["H0"]) < 1e-9 * abs(i64["H0"])
    assert abs(i64["plaquette"] - imx["plaquette"]) < 1e-12
    assert rel(o64, omx) < 1e-10
    d.close()
