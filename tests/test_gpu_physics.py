"""Physics checks on the GPU against the float64 CPU oracle.

* Static bubble (64^3 periodic box, radius 16, tau 0.8, sigma 0.01, beta 0.7,
  2000 steps): the float32 solver against the float64 oracle from the same
  seeded state (max |d psi| <= 1e-3, Laplace jump within 2 %, spurious-current
  peak within 5 %), and Laplace's law dp * R_eff constant across radii.
* Float16 storage: the 64x128x64 jet crop run in float32 and float16 storage
  against the float64 oracle, at D=8 (y/D = 2..6 inside the crop) and at the
  256x512x256 jet's D=32 (Re 240, We 16: the same tau 0.52 and sigma 0.005;
  y/D = 1..3); the radial mean centre-line velocity and half-width agree
  within 1 % (the bar float16 storage is held to).
"""
import numpy as np
import pytest

from helpers import interior, maxabs, psi_of
from multicomponent_color_gradient_b200 import Solver, get_case
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def _interior_grid(F, case, key):
    NX, NY, NZ = case["NX"], case["NY"], case["NZ"]
    return np.asarray(F[key], np.float64).reshape(NZ, NY, NX)[1:-1, 1:-1, 1:-1]


def test_static_bubble_fp32_vs_fp64_oracle_and_laplace():
    case = get_case("bubble_64")
    S = Solver(case)
    S.init_bubble()
    fr, fb = S.get_populations()
    F0 = S.get_fields()
    O = Oracle(case, 64)
    O.set_fields(F0["rhor"], F0["rhob"], F0["ux"], F0["uy"], F0["uz"])
    O.set_populations(fr, fb)
    S.step(2000)
    O.step(2000)
    F, OF = S.get_fields(), O.get_fields()
    m = interior(case)
    dpsi = maxabs(psi_of(F["rhor"][m], F["rhob"][m]), psi_of(OF["rhor"][m], OF["rhob"][m]))
    umax = np.sqrt(F["ux"][m] ** 2 + F["uy"][m] ** 2 + F["uz"][m] ** 2).max()
    oumax = np.sqrt(OF["ux"][m] ** 2 + OF["uy"][m] ** 2 + OF["uz"][m] ** 2).max()
    dp, odp = laplace_jump(F, case), laplace_jump(OF, case)
    print(f"bubble 64^3 R=16: dp={dp:.4e} (fp64 {odp:.4e}; 2 sigma/R_eff = {2 * case['sigma'] / r_eff(F, case):.4e}),"
          f" spurious |u|max={umax:.3e} (fp64 {oumax:.3e}), max|d psi|={dpsi:.2e}")
    assert dpsi <= 1e-3, dpsi
    # Laplace jump (p = cs^2 rho) and spurious-current peak against the float64 oracle's
    assert abs(dp - odp) <= 0.02 * abs(odp)
    assert umax < 5e-3
    assert abs(umax - oumax) <= 0.05 * oumax + 1e-6, (umax, oumax)


def laplace_jump(F, case):
    rho = _interior_grid(F, case, "rhor") + _interior_grid(F, case, "rhob")
    c = rho.shape[0] // 2
    p_in = rho[c - 3:c + 3, c - 3:c + 3, c - 3:c + 3].mean() / 3.0
    p_out = rho[:4, :4, :4].mean() / 3.0
    return p_in - p_out


def r_eff(F, case):
    """Radius of the sphere with the drop's volume, V = sum (1 + psi_drop) / 2."""
    rr, rb = _interior_grid(F, case, "rhor"), _interior_grid(F, case, "rhob")
    inside = (rr if case.get("bubble_red_inside", 0) else rb) / (rr + rb)
    return float((3.0 * inside.sum() / (4.0 * np.pi)) ** (1.0 / 3.0))


def test_laplace_law_scaling():
    """dp * R_eff is the same for two drop radii (Laplace's law, dp = 2 sigma_eff / R).
    The colour-gradient operator as the reference calibrates it (A = sigma /
    (4 cs^4 tau) on the gradient of psi in [-1,1]) gives sigma_eff below the
    input sigma on this lattice; the ratio is reported and bounded loosely."""
    res = {}
    for R in (12.0, 18.0):
        case = get_case("bubble_64", bubble_radius=R, init_noise=0.0)
        S = Solver(case)
        S.init_bubble()
        S.step(1500)
        F = S.get_fields()
        res[R] = laplace_jump(F, case) * r_eff(F, case) / 2
    sigma = get_case("bubble_64")["sigma"]
    print(f"sigma_eff(R=12)={res[12.0]:.4e} sigma_eff(R=18)={res[18.0]:.4e} input sigma={sigma}")
    # measured: 4.90e-3 and 4.17e-3 (interface ~4-5 nodes wide, periodic images 26 nodes apart)
    assert abs(res[12.0] - res[18.0]) <= 0.25 * res[18.0]
    assert 0.3 * sigma < res[18.0] < 1.5 * sigma


def radial_mean_uy(R, NY, NRB):
    cnt = R["count"].astype(np.float64).reshape(NY, NRB)
    s = R["sum_uy"].reshape(NY, NRB)
    out = np.full_like(s, np.nan)
    np.divide(s, cnt, out=out, where=cnt > 0)
    return out


def half_width(profile, radius):
    """First radius where u/u_c falls to 1/2 (linear interpolation, as the
    post-processing of the radial profiles does)."""
    uc = profile[0]
    ratio = profile / uc
    below = np.where(np.isfinite(ratio) & (ratio <= 0.5))[0]
    below = below[below > 0]
    if below.size == 0 or not np.isfinite(uc) or uc <= 0:
        return np.nan
    k = int(below[0])
    r1, r2, u1, u2 = radius[k - 1], radius[k], ratio[k - 1], ratio[k]
    return r1 + (0.5 - u1) * (r2 - r1) / (u2 - u1)


def bin_centres(case):
    NX, NZ, NRB = case["NX"], case["NZ"], case["NX"] // 2
    x = np.arange(1, NX - 1, dtype=np.float32) - np.float32(case["jet_x0"])
    z = np.arange(1, NZ - 1, dtype=np.float32) - np.float32(case["jet_z0"])
    r = np.sqrt((x[None, :] ** 2 + z[:, None] ** 2).astype(np.float32)).astype(np.float64)
    rb = r.astype(np.int64)
    sums = np.bincount(rb.ravel(), weights=r.ravel(), minlength=NRB)[:NRB]
    cnts = np.bincount(rb.ravel(), minlength=NRB)[:NRB]
    out = np.arange(NRB, dtype=np.float64)
    np.divide(sums, cnts, out=out, where=cnts > 0)
    out[0] = 0.0
    return out


# Crop runs: (diameter D, steps, statistics from, rows as multiples of D).
# D=8 is the crop scaled with the domain; D=32 keeps the 256x512x256 jet's
# own diameter (Re 240, We 16 give the same tau 0.52 and sigma 0.005), so the
# crop holds y/D <= 4 and the jet fills half the lateral width.
CROPS = {
    8: dict(steps=1200, stats_from=600, overrides={}, ks=(2, 3, 4, 5, 6)),
    32: dict(steps=2400, stats_from=1200, overrides=dict(jet_radius=16.0, Re=240.0, We=16.0), ks=(1, 2, 3)),
}
_crop_oracle = {}


def _crop_case(D, **kw):
    c = CROPS[D]
    return get_case("jet_64x128x64", NSTATS_START_STEP=c["stats_from"], **c["overrides"], **kw)


def _crop_oracle_run(D):
    """The float64 oracle's radial statistics and fields of crop D (one run
    shared by both storages)."""
    if D not in _crop_oracle:
        O = Oracle(_crop_case(D), 64)
        O.init_jet()
        O.step(CROPS[D]["steps"])
        _crop_oracle[D] = (O.get_radial(), O.get_fields())
    return _crop_oracle[D]


@pytest.mark.parametrize("D", [8, 32])
@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_jet_crop_profiles_within_one_percent_of_fp64(storage, D):
    case = _crop_case(D, storage=storage)
    assert 2 * case["jet_radius"] == D
    if D == 32:
        assert abs(case["taur"] - 0.52) < 1e-6 and abs(case["sigma"] - 0.005) < 1e-6, (case["taur"], case["sigma"])
    S = Solver(case)
    S.init_jet()
    S.step(CROPS[D]["steps"])
    OR, OF = _crop_oracle_run(D)
    NY, NRB = case["NY"], case["NX"] // 2
    U, OU = radial_mean_uy(S.get_radial(), NY, NRB), radial_mean_uy(OR, NY, NRB)
    radius = bin_centres(case)
    rows = [int(round(k * D)) for k in CROPS[D]["ks"]]
    for y in rows:
        uc, ouc = U[y, 0], OU[y, 0]
        assert abs(uc - ouc) <= 0.01 * abs(ouc), (storage, D, y, uc, ouc)
        hw, ohw = half_width(U[y], radius), half_width(OU[y], radius)
        if np.isfinite(ohw):
            assert abs(hw - ohw) <= 0.01 * ohw, (storage, D, y, hw, ohw)
        print(f"{storage} D={D} y/D={y / D:.0f}: u_c {uc:.6f} (fp64 {ouc:.6f}), r_half {hw:.4f} (fp64 {ohw:.4f})")
    F = S.get_fields()
    S.close()
    m = interior(case)
    dpsi = maxabs(psi_of(F["rhor"][m], F["rhob"][m]), psi_of(OF["rhor"][m], OF["rhob"][m]))
    print(f"{storage} D={D}: max|d psi| vs fp64 = {dpsi:.3e}")
    assert dpsi <= (1e-3 if storage == "f32" else 2e-2)
