"""Parity of the CUDA step with the CPU oracle and with the reference's own CUDA build.

Tolerances (float32 arithmetic on both sides; the reference and this solver
contract multiply-adds differently, so results agree to rounding, not bits):
  populations after 100 steps from the same state:  max-abs <= 2e-5
  macroscopic fields / stress:                       max-abs <= 2e-5
  radial float64 sums:                               |d sum| <= 2e-5 * count per bin
                                                     (the field tolerance per sample)
Radial counts are integers and must match exactly.  The granular launch
sequence and the fused step compute the boundary values in different kernels,
whose multiply-add contraction may differ, so they agree to 1e-6, not bits.
"""
import numpy as np
import pytest

from helpers import initial_state, interior, maxabs, pops_interior, psi_of, run_reference
from conftest import ref_binary
from multicomponent_color_gradient_b200 import Solver, get_case
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

POP_ATOL = 2e-5
FIELD_ATOL = 2e-5
SAMPLE_ATOL = 2e-5

SMALL = [("bubble_24_ref", 100, 10**9, 1e-6), ("jet_24x40x24", 100, 20, 1e-6), ("jet_32x48x32", 100, 20, 0.0)]


def _solver_from_state(case, state):
    fr, fb, fields = state
    S = Solver(case)
    S.set_fields(**fields)
    S.set_populations(fr, fb)
    return S


def _oracle_from_state(case, state, precision):
    fr, fb, fields = state
    O = Oracle(case, precision)
    O.set_fields(**fields)
    O.set_populations(fr, fb)
    return O


def _radial_close(a, b, atol=SAMPLE_ATOL):
    np.testing.assert_array_equal(a["count"], b["count"])
    cnt = np.maximum(np.asarray(b["count"], np.float64), 1.0)
    for k in ("sum_uy", "sum_uy2", "sum_ur", "sum_ur2", "sum_uruy"):
        err = np.max(np.abs(a[k] - b[k]) / cnt)
        assert err <= atol, (k, err)


@pytest.mark.parametrize("name,steps,stats_from,noise", SMALL)
@pytest.mark.parametrize("precision", [32, 64])
def test_step_matches_oracle(name, steps, stats_from, noise, precision):
    case = get_case(name, NSTATS_START_STEP=stats_from)
    state = initial_state(case, noise=noise, seed=7)
    S = _solver_from_state(case, state)
    O = _oracle_from_state(case, state, precision)
    S.step(steps)
    O.step(steps)
    assert S.current_step == O.current_step == steps
    fr, fb = S.get_populations()
    ofr, ofb = O.get_populations()
    e_r = maxabs(pops_interior(fr, case), pops_interior(ofr, case))
    e_b = maxabs(pops_interior(fb, case), pops_interior(ofb, case))
    m = interior(case)
    F, OF = S.get_fields(), O.get_fields()
    errs = {k: maxabs(F[k][m], OF[k][m]) for k in ("rhor", "rhob", "ux", "uy", "uz")}
    print(f"{name} fp{precision}: pops r {e_r:.3e} b {e_b:.3e} fields {errs}")
    assert e_r <= POP_ATOL and e_b <= POP_ATOL, (e_r, e_b)
    for k, e in errs.items():
        assert e <= FIELD_ATOL, (k, e)
    assert maxabs(S.get_stress().reshape(6, -1)[:, m], O.get_stress().reshape(6, -1)[:, m]) <= FIELD_ATOL
    if case["boundary"] == "jet":
        # outlet state on y = NY-1 (jet/boundary_conditions.cuh:184-196)
        NX, NY, NZ = case["NX"], case["NY"], case["NZ"]
        sel = np.zeros((NZ, NY, NX), bool)
        sel[1:-1, NY - 1, 1:-1] = True
        sel = sel.reshape(-1)
        for k in ("rhor", "rhob", "ux", "uy", "uz"):
            assert maxabs(F[k][sel], OF[k][sel]) <= FIELD_ATOL, ("outlet", k)
        assert S.radial_state() == O.radial_state()
        _radial_close(S.get_radial(), O.get_radial())


@pytest.mark.parametrize("name,steps,stats_from,noise", SMALL)
def test_granular_sequence_equals_fused_step(name, steps, stats_from, noise):
    """launch_Macros/accumulate/collistream/inlet/neumann == the fused step."""
    case = get_case(name, NSTATS_START_STEP=stats_from)
    state = initial_state(case, noise=noise, seed=3)
    A = _solver_from_state(case, state)
    B = _solver_from_state(case, state)
    A.step(steps)
    for s in range(steps):
        B.launch_Macros()
        if s >= stats_from:
            B.launch_accumulate_radial_moments()
        B.launch_collistream()
        if case["boundary"] == "jet":
            B.launch_inlet_bc()
            B.launch_neumann_bc()
    fa, fb_ = A.get_populations()
    ga, gb = B.get_populations()
    assert maxabs(fa, ga) <= 1e-6 and maxabs(fb_, gb) <= 1e-6
    Fa, Fb = A.get_fields(), B.get_fields()
    for k in Fa:
        assert maxabs(Fa[k], Fb[k]) <= 1e-6, k
    if case["boundary"] == "jet":
        _radial_close(A.get_radial(), B.get_radial(), atol=1e-6)
        assert A.radial_state() == B.radial_state()


@pytest.mark.parametrize("name", ["bubble_24_ref", "jet_24x40x24", "bubble_64"])
def test_population_roundtrip(name):
    case = get_case(name)
    fr, fb, fields = initial_state(case, noise=1e-3, seed=11)
    S = _solver_from_state(case, (fr, fb, fields))
    gr, gb = S.get_populations()
    np.testing.assert_array_equal(pops_interior(gr, case), pops_interior(fr, case))
    np.testing.assert_array_equal(pops_interior(gb, case), pops_interior(fb, case))
    # ghost nodes are reported as zero
    assert not np.any(gr.reshape(27, -1)[:, ~interior(case)])


@pytest.mark.parametrize("name,steps,stats_from", [("bubble_24_ref", 100, 10**9), ("jet_24x40x24", 100, 20),
                                                   ("jet_32x48x32", 100, 20)])
def test_matches_reference_build_small(name, steps, stats_from):
    if ref_binary(name) is None:
        pytest.skip("reference build oracle/_ref/ref_%s not present" % name)
    case = get_case(name)
    state = initial_state(case, noise=1e-6 if case["boundary"] != "jet" else 0.0, seed=5)
    R = run_reference(name, case, steps, stats_from, state=state)
    # the reference driver starts statistics at stats_from; so does NSTATS_START_STEP
    S2 = Solver(get_case(name, NSTATS_START_STEP=stats_from))
    S2.set_fields(**state[2])
    S2.set_populations(state[0], state[1])
    S2.step(steps)
    fr, fb = S2.get_populations()
    assert maxabs(pops_interior(fr, case), pops_interior(R["fr"], case)) <= POP_ATOL
    assert maxabs(pops_interior(fb, case), pops_interior(R["fb"], case)) <= POP_ATOL
    F = S2.get_fields()
    m = interior(case)
    for k in ("rhor", "rhob", "ux", "uy", "uz"):
        assert maxabs(F[k][m], R[k][m]) <= FIELD_ATOL, k
    if case["boundary"] == "jet":
        _radial_close(S2.get_radial(), R)


@pytest.mark.parametrize("name,stats_from", [("bubble_64_ref", 10**9), ("jet_128x256x128", 50)])
def test_matches_reference_build_full_size(name, stats_from):
    """The full-size workloads (bubble 64^3, jet 128x256x128), 100 steps from each code's own initial condition:
    max-abs on populations and on psi (the parity measure of the step)."""
    if ref_binary(name) is None:
        pytest.skip("reference build oracle/_ref/ref_%s not present" % name)
    case = get_case(name, NSTATS_START_STEP=stats_from)
    steps = 100
    R = run_reference(name, case, steps, stats_from)
    S = Solver(case)
    if case["boundary"] == "jet":
        S.init_jet()
    else:
        S.init_bubble()
    S.step(steps)
    fr, fb = S.get_populations()
    e_r = maxabs(pops_interior(fr, case), pops_interior(R["fr"], case))
    e_b = maxabs(pops_interior(fb, case), pops_interior(R["fb"], case))
    F = S.get_fields()
    m = interior(case)
    e_psi = maxabs(psi_of(F["rhor"][m], F["rhob"][m]), psi_of(R["rhor"][m], R["rhob"][m]))
    print(f"{name}: max|dfr|={e_r:.3e} max|dfb|={e_b:.3e} max|dpsi|={e_psi:.3e}")
    assert e_r <= POP_ATOL and e_b <= POP_ATOL
    assert e_psi <= 1e-4
    if case["boundary"] == "jet":
        _radial_close(S.get_radial(), R)


def test_periodic_bubble_conserves_each_colour():
    case = get_case("bubble_64", NSTEP=200)
    S = Solver(case)
    S.init_bubble()
    s0 = S.conservation_sums()
    S.step(200)
    s1 = S.conservation_sums()
    assert abs(s1[0] - s0[0]) / s0[0] < 2e-6
    assert abs(s1[1] - s0[1]) / s0[1] < 2e-6
    assert S.check_finite()


def test_periodic_bubble_matches_oracle():
    case = get_case("bubble_64")
    S = Solver(case)
    S.init_bubble()
    fr, fb = S.get_populations()
    F = S.get_fields()
    O = Oracle(case, 64)
    O.set_fields(F["rhor"], F["rhob"], F["ux"], F["uy"], F["uz"])
    O.set_populations(fr, fb)
    # the oracle's periodic ghost densities are refreshed from the interior
    S.step(50)
    O.step(50)
    a, b = S.get_populations()
    oa, ob = O.get_populations()
    assert maxabs(pops_interior(a, case), pops_interior(oa, case)) <= POP_ATOL
    assert maxabs(pops_interior(b, case), pops_interior(ob, case)) <= POP_ATOL


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("name", ["jet_24x40x24", "bubble_64"])
@pytest.mark.parametrize("pipe", ["0", "1"])
@pytest.mark.parametrize("nx", [128, 256])
def test_fixed_row_length_kernels_equal_runtime_geometry(monkeypatch, storage, name, pipe, nx):
    """Rows of exactly 128 or 256 columns run fused kernels compiled for that
    row length (constant slot and row offsets); they produce the populations
    and fields of the runtime-geometry kernels bit for bit, in both marches."""
    case = get_case(name, NX=nx, NY=24, NZ=22, storage=storage, NSTATS_START_STEP=0)
    state = initial_state(case, noise=1e-3 if case["boundary"] != "jet" else 0.0, seed=13)
    monkeypatch.setenv("MCG_FUSED_PIPE", pipe)
    out = []
    for fixed in ("1", "0"):
        monkeypatch.setenv("MCG_FUSED_FIXED_NX", fixed)
        with _solver_from_state(case, state) as S:
            assert S.tiling()["fixed_row_length"] == (nx if fixed == "1" else 0)
            S.step(30)
            out.append((S.get_populations(), S.get_fields()))
    (pa, fa), (pb, fb) = out
    np.testing.assert_array_equal(pa[0], pb[0])
    np.testing.assert_array_equal(pa[1], pb[1])
    for k in fa:
        np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("name,shape", [("jet_24x40x24", (40, 32, 36)), ("bubble_64", (72, 20, 34))])
def test_pipelined_march_equals_block_synchronous_march(monkeypatch, storage, name, shape):
    """k_fused_pipe (one barrier per plane; float16 with its loads in flight
    across another row's relaxation) and k_fused (two barriers per plane) do
    the same arithmetic in the same order: equal populations and fields, bit
    for bit, on row lengths other than 128 (64 and 96 threads per row, idle
    lanes included) and 16-plane chunks."""
    NX, NY, NZ = shape
    case = get_case(name, NX=NX, NY=NY, NZ=NZ, storage=storage, NSTATS_START_STEP=0)
    state = initial_state(case, noise=1e-3 if case["boundary"] != "jet" else 0.0, seed=17)
    monkeypatch.setenv("MCG_FUSED_LZ", "16")
    out = []
    for pipe in ("1", "0"):
        monkeypatch.setenv("MCG_FUSED_PIPE", pipe)
        with _solver_from_state(case, state) as S:
            t = S.tiling()
            assert t["pipelined"] == int(pipe) and t["fixed_row_length"] == 0
            S.step(25)
            out.append((S.get_populations(), S.get_fields(), S.get_radial() if case["boundary"] == "jet" else None))
    (pa, fa, ra), (pb, fb, rb) = out
    np.testing.assert_array_equal(pa[0], pb[0])
    np.testing.assert_array_equal(pa[1], pb[1])
    for k in fa:
        np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)
    if case["boundary"] == "jet":
        _radial_close(ra, rb, atol=1e-9)


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("name,shape", [("jet_24x40x24", (128, 40, 60)), ("bubble_64", (100, 30, 40)),
                                        ("jet_24x40x24", (256, 20, 36))])
def test_marches_agree_bit_for_bit(monkeypatch, storage, name, shape):
    """The block-synchronous and the pipelined march give equal populations
    and fields, bit for bit, on 128-, 100- and 256-column rows, both
    storages, jet and periodic box, 16-plane chunks."""
    NX, NY, NZ = shape
    case = get_case(name, NX=NX, NY=NY, NZ=NZ, storage=storage, NSTATS_START_STEP=0)
    state = initial_state(case, noise=1e-3 if case["boundary"] != "jet" else 0.0, seed=29)
    out = []
    for pipe in ("0", "1"):
        monkeypatch.setenv("MCG_FUSED_PIPE", pipe)
        monkeypatch.setenv("MCG_FUSED_LZ", "16")
        with _solver_from_state(case, state) as S:
            t = S.tiling()
            assert t["pipelined"] == int(pipe)
            S.step(20)
            out.append((S.get_populations(), S.get_fields(), S.get_radial() if case["boundary"] == "jet" else None,
                        t))
    ref = out[0]
    for other in out[1:]:
        np.testing.assert_array_equal(other[0][0], ref[0][0], err_msg=str(other[3]))
        np.testing.assert_array_equal(other[0][1], ref[0][1], err_msg=str(other[3]))
        for k in ref[1]:
            np.testing.assert_array_equal(other[1][k], ref[1][k], err_msg=k)
        if case["boundary"] == "jet":
            _radial_close(other[2], ref[2], atol=1e-9)


def _march(monkeypatch, case, state, steps, bulk, lz="16"):
    """Populations, fields and radial sums after `steps` steps of the pipelined
    march, with (bulk) or without rows staged by bulk copies."""
    monkeypatch.setenv("MCG_FUSED_PIPE", "1")
    monkeypatch.setenv("MCG_FUSED_BULK", "1" if bulk else "0")
    monkeypatch.setenv("MCG_FUSED_LZ", lz)
    with _solver_from_state(case, state) as S:
        t = S.tiling()
        assert t["pipelined"] == (2 if bulk else 1), t
        S.step(steps)
        S.synchronize()
        return (S.get_populations(), S.get_fields(),
                S.get_radial() if case["boundary"] == "jet" else None, t)


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("name,shape,lz", [("jet_24x40x24", (128, 40, 60), "16"),
                                           ("jet_24x40x24", (128, 23, 19), "5"),
                                           ("bubble_64", (128, 30, 40), "16")])
def test_bulk_staged_march_is_bit_identical(monkeypatch, storage, name, shape, lz):
    """k_fused_bulk (each pulled row's 9 source segments staged in shared
    memory by cp.async.bulk) gives the populations, fields and radial sums of
    k_fused_pipe bit for bit: jet with its ghost rows and planes, a grid whose
    last tile and chunk are partial, the periodic box with its wrapped rows."""
    NX, NY, NZ = shape
    case = get_case(name, NX=NX, NY=NY, NZ=NZ, storage=storage, NSTATS_START_STEP=0)
    state = initial_state(case, noise=1e-3 if case["boundary"] != "jet" else 0.0, seed=31)
    ref = _march(monkeypatch, case, state, 20, bulk=False, lz=lz)
    got = _march(monkeypatch, case, state, 20, bulk=True, lz=lz)
    np.testing.assert_array_equal(got[0][0], ref[0][0], err_msg=str(got[3]))
    np.testing.assert_array_equal(got[0][1], ref[0][1], err_msg=str(got[3]))
    for k in ref[1]:
        np.testing.assert_array_equal(got[1][k], ref[1][k], err_msg=k)
    if case["boundary"] == "jet":
        _radial_close(got[2], ref[2], atol=1e-9)


def test_bulk_staged_wait_limit_reports_timeout(monkeypatch):
    """With a wait limit of 0 tries every wait for a staged row runs out: the
    kernel flags it, drains its copies in flight and returns, and the next
    synchronisation reports MCG_ERR_TIMEOUT.  The handle stays usable: with the
    default limit restored and the state set again, further steps match the
    pipelined march run through the same sequence of calls."""
    from multicomponent_color_gradient_b200._lib import McgError

    case = get_case("jet_24x40x24", NX=128, NY=40, NZ=60, NSTATS_START_STEP=0)
    state = initial_state(case, noise=0.0, seed=37)
    fr, fb, fields = state
    monkeypatch.setenv("MCG_FUSED_PIPE", "1")
    monkeypatch.setenv("MCG_FUSED_LZ", "16")
    out = {}
    for bulk in (False, True):
        monkeypatch.setenv("MCG_FUSED_BULK", "1" if bulk else "0")
        with _solver_from_state(case, state) as S:
            assert S.tiling()["pipelined"] == (2 if bulk else 1)
            if bulk:
                S.set_stage_wait_limit(0)
                S.step(3)
                with pytest.raises(McgError) as err:
                    S.synchronize()
                assert err.value.status == 6  # MCG_ERR_TIMEOUT
                S.synchronize()  # the flag was cleared
                S.set_stage_wait_limit(1 << 20)
            else:
                S.step(3)
                S.synchronize()
            S.set_fields(**fields)
            S.set_populations(fr, fb)
            S.step(6)
            S.synchronize()
            out[bulk] = S.get_populations()
    np.testing.assert_array_equal(out[True][0], out[False][0])
    np.testing.assert_array_equal(out[True][1], out[False][1])


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("march", ["0", "1", "bulk"])
@pytest.mark.parametrize("shape", [(128, 40, 60), (100, 30, 40)])
def test_boundary_in_the_fused_step_equals_the_boundary_launch(monkeypatch, storage, march, shape):
    """The jet's inlet and outlet columns written by the fused step's own-row
    threads of rows 1 and NY-2 equal those of a separate k_boundary launch
    after the step, bit for bit: populations, fields (the outlet's carried
    state and the inlet mask included) and radial sums, with the seeded inlet
    perturbation, in every march and both storages."""
    NX, NY, NZ = shape
    if march == "bulk" and NX != 128:
        pytest.skip("the bulk-staged march runs 128-column rows")
    case = get_case("jet_24x40x24", NX=NX, NY=NY, NZ=NZ, storage=storage, NSTATS_START_STEP=0,
                    inlet_noise=0.01, seed=5)
    state = initial_state(case, noise=0.0, seed=41)
    monkeypatch.setenv("MCG_FUSED_PIPE", "0" if march == "0" else "1")
    monkeypatch.setenv("MCG_FUSED_BULK", "1" if march == "bulk" else "0")
    monkeypatch.setenv("MCG_FUSED_LZ", "8")
    out = []
    for fused in ("1", "0"):
        monkeypatch.setenv("MCG_FUSED_BOUNDARY", fused)
        with _solver_from_state(case, state) as S:
            l0 = S.launches
            S.step(12)
            launches = S.launches - l0
            out.append((S.get_populations(), S.get_fields(), S.get_radial(), launches))
    (pa, fa, ra, la), (pb, fb, rb, lb) = out
    assert (la, lb) == (12, 24)
    np.testing.assert_array_equal(pa[0], pb[0])
    np.testing.assert_array_equal(pa[1], pb[1])
    for k in fa:
        np.testing.assert_array_equal(fa[k], fb[k], err_msg=k)
    _radial_close(ra, rb, atol=1e-9)
