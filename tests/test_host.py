"""CPU: host set-up code of the library (graph, tables, config, masks) and
the C ABI library itself (exports, admission checks that need no GPU)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import heom_b200 as hb
import heom_oracle as ho

from conftest import gpu_available

FMO_CFG = """[program]
task=population_dynamics
observations={(matrix_complete, m.dat), (matrix_diagonal, d.dat), (matrix_trace_id, t.dat)}
observe_steps=5

[filtering]
strategy=none
first_layer=-1

[solver]
stepper_type=rk_rk4
step_size=1.0e-15
steps=20
track_flows=false
flow_filename=

[system]
sites=3
hamiltonian={{12410.0, -87.7, 5.5}, {-87.7, 12530.0, 30.8}, {5.5, 30.8, 12210.0}}
ado_depth=3

[baths]
number=3
max_per_site=1
coupling={{0}, {1}, {2}}
lambda={35, 35, 35}
invnu={50, 50, 50}
Omega={0, 0, 0}
matsubaras=2
temperature=77 # K

[population_dynamics]
rho_init={{1.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}}
"""


def header_functions(root):
    src = open(os.path.join(root, "include", "heom_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(heom_\w+)\s*\(", src)))


def test_library_exports_every_header_symbol(root):
    names = header_functions(root)
    assert sorted(hb.EXPORTS) == names
    L = C.CDLL(hb.LIB_PATH)
    for n in names:
        assert hasattr(L, n), n


@pytest.mark.parametrize("n,d,m,seed", [(7, 4, 1, 11), (8, 3, 2, 22), (5, 3, 3, 5), (2, 6, 1, 1)])
def test_tables_identical_to_oracle(n, d, m, seed):
    h = ho.synthetic_hamiltonian(n, seed)
    prob = ho.build_problem(ho.make_system(h, [35.0] * n, [50.0] * n, [0.0] * n, m, 300.0, d))
    t = hb.build_tables(hb.System(h, [35.0] * n, [50.0] * n, [0.0] * n, m, 300.0, d))
    g = prob.graph
    assert t["matrices"] == g.nodes and t["first_non_plus_id"] == g.first_non_plus
    for k, v in [("ado_tuples", g.tuples), ("ado_plus", g.plus), ("ado_minus", g.minus),
                 ("pf_same_sum", prob.pf_same_sum), ("pf_same", prob.pf_same), ("pf_circ", prob.pf_circ),
                 ("cbk", prob.cbk), ("cbk_sqrt", prob.cbk_sqrt), ("hamiltonian", prob.hamiltonian)]:
        assert np.array_equal(t[k], np.asarray(v).reshape(-1)), k


def test_tables_omega_and_shared_coupling():
    h = ho.synthetic_hamiltonian(3, 8)
    cpl = np.array([[0, 1], [1, 2], [2, -1]], np.int32)
    lam, inv, om = [35, 25, 45], [50, 45, 65], [0.0, 15.0, -15.0]
    prob = ho.build_problem(ho.make_system(h, lam, inv, om, 2, 280.0, 3, coupling=cpl))
    t = hb.build_tables(hb.System(h, lam, inv, om, 2, 280.0, 3, coupling=cpl))
    for k, v in [("pf_same_sum", prob.pf_same_sum), ("pf_same", prob.pf_same), ("pf_circ", prob.pf_circ),
                 ("cbk", prob.cbk), ("cbk_sqrt", prob.cbk_sqrt)]:
        assert np.array_equal(t[k], v), k


def test_config_parses_reference_style_file(tmp_path):
    p = tmp_path / "a.cfg"
    p.write_text(FMO_CFG)
    c = hb.Config(p)
    assert c.get("solver.stepper_type") == "rk_rk4"
    d = c.system_desc()
    assert d.sites == 3 and d.ado_depth == 3 and d.matsubaras == 2 and d.temperature == 77.0
    r = c.rho_init()
    assert r[0] == 1.0 and r[1:].sum() == 0.0


@pytest.mark.parametrize("edit,msg", [
    (("steps=20", "steps=21"), "remainder"),
    (("strategy=none", "strategy=bogus"), "filtering"),
    (("first_layer=-1", "first_layer=0"), "first_layer"),
    (("{-87.7, 12530.0, 30.8}", "{-87.0, 12530.0, 30.8}"), "hermitian"),
    (("sites=3", "sites=4"), "matrix"),
    (("task=population_dynamics", "task=thermal_state_search"), "program.task"),
    (("task=population_dynamics", "task=linear_absorption"), "population_dynamics.rho_init"),
    (("stepper_type=rk_rk4", "stepper_type=rk_euler"), "rk_rk4"),
    (("lambda={35, 35, 35}", "lambda={35, 35}"), "lambda"),
    (("invnu={50, 50, 50}", "invnu={50, 0, 50}"), "invnu"),
    (("coupling={{0}, {1}, {2}}", "coupling={{0}, {1}, {3}}"), "coupling"),
    (("observe_steps=5", "observe_steps=5\nbogus_key=1"), "unrecognised"),
    (("matsubaras=2", "matsubaras=11"), "matsubaras"),
])
def test_config_rejects_invalid(tmp_path, edit, msg):
    p = tmp_path / "bad.cfg"
    p.write_text(FMO_CFG.replace(*edit))
    with pytest.raises(hb.HeomError) as e:
        hb.Config(p)
    assert msg in str(e.value)


LA_CFG = FMO_CFG.replace("task=population_dynamics", "task=linear_absorption").replace(
    "observations={(matrix_complete, m.dat), (matrix_diagonal, d.dat), (matrix_trace_id, t.dat)}",
    "observations={(matrix_trace_linear_absorption, la.dat)}").split("[population_dynamics]")[0] + """[dipole]
directions={{-0.741, -0.561, -0.370}, {-0.857, 0.504, -0.107}, {-0.197, 0.957, -0.211}}
centers={{2.651, 0.260, -1.135}, {1.561, -0.152, -1.725}, {0.339, -1.361, -1.385}}
strengths={4, 3.5, 4.2}
tensor_prefactors={1, 1, 1}
tensor_components={{0, 0}, {1, 1}, {2, 2}}
"""


def test_linear_absorption_config(tmp_path):
    p = tmp_path / "la.cfg"
    p.write_text(LA_CFG)
    c = hb.Config(p)
    assert c.get("program.task") == "linear_absorption"
    assert c.get("dipole.strengths") == "{4, 3.5, 4.2}"
    with pytest.raises(hb.HeomError):
        c.rho_init()  # a population_dynamics entry
    # dipole entries belong to the linear_absorption task only, and must agree in size
    p.write_text(FMO_CFG + LA_CFG.split("[baths]")[1].split("temperature=77 # K")[1])
    with pytest.raises(hb.HeomError) as e:
        hb.Config(p)
    assert "unrecognised option 'dipole." in str(e.value)
    p.write_text(LA_CFG.replace("strengths={4, 3.5, 4.2}", "strengths={4, 3.5}"))
    with pytest.raises(hb.HeomError) as e:
        hb.Config(p)
    assert "same size" in str(e.value)
    p.write_text(LA_CFG.replace("tensor_prefactors={1, 1, 1}", "tensor_prefactors={1, 1}"))
    with pytest.raises(hb.HeomError) as e:
        hb.Config(p)
    assert "same size" in str(e.value)


def test_linear_absorption_app_reports_config_errors_before_the_device(tmp_path, root):
    app = os.path.join(root, "dm-heom_b200", "bin", "heom_linear_absorption")
    (tmp_path / "rt.cfg").write_text("[cuda]\ndevice_index=0\n")
    (tmp_path / "pd.cfg").write_text(FMO_CFG)
    r = subprocess.run([app, "rt.cfg", "pd.cfg"], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "population_dynamics.rho_init" not in r.stderr
    assert "wrong program_task" in r.stderr
    (tmp_path / "la.cfg").write_text(LA_CFG.replace("tensor_components={{0, 0}, {1, 1}, {2, 2}}",
                                                    "tensor_components={{0, 0}, {1, 1}, {2, 5}}"))
    r = subprocess.run([app, "rt.cfg", "la.cfg"], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "out of range" in r.stderr


def test_circular_dichroism_config_and_app_tasks(tmp_path, root):
    cd = LA_CFG.replace("task=linear_absorption", "task=circular_dichroism")
    (tmp_path / "cd.cfg").write_text(cd)
    assert hb.Config(tmp_path / "cd.cfg").get("program.task") == "circular_dichroism"
    (tmp_path / "la.cfg").write_text(LA_CFG)
    (tmp_path / "rt.cfg").write_text("[cuda]\ndevice_index=0\n")
    bins = os.path.join(root, "dm-heom_b200", "bin")
    for app, cfg in (("heom_circular_dichroism", "la.cfg"), ("heom_linear_absorption", "cd.cfg")):
        r = subprocess.run([os.path.join(bins, app), "rt.cfg", cfg], cwd=tmp_path, capture_output=True,
                           text=True, timeout=60)
        assert r.returncode != 0 and "wrong program_task" in r.stderr


def test_config_missing_file():
    with pytest.raises(hb.HeomError):
        hb.Config("/nonexistent/file.cfg")


def test_single_excitation_mask_matches_restatement():
    import make_golden as mg
    s = hb.System(ho.synthetic_hamiltonian(4, 1), [35] * 4, [50] * 4, [0] * 4, 2, 300.0, 3)
    m = hb.tables_mask(s, "single_excitation", 1)
    g = ho.build_graph(8, 3)
    assert np.array_equal(m, mg.single_excitation_mask(g, 2, 1))
    assert (hb.tables_mask(s, "none", -1) == 1).all()


def _good_desc():
    h = ho.synthetic_hamiltonian(3, 2)
    return hb.build_tables(hb.System(h, [35] * 3, [50] * 3, [0] * 3, 1, 300.0, 2))


@pytest.mark.parametrize("field,index,value,code", [
    ("ado_plus", 0, 999, -4), ("ado_minus", 5, -7, -4), ("ado_tuples", 3, 9, -4),
    ("baths_coupling", 0, 7, -4)])
def test_admission_rejects_bad_tables(field, index, value, code):
    # table admission runs before any CUDA call, so it is testable on the CPU
    d = _good_desc()
    d[field] = d[field].copy()
    d[field][index] = value
    with pytest.raises(hb.HeomError) as e:
        hb.Heom(**d)
    assert f"heom error {code}" in str(e.value)


def test_admission_rejects_sizes():
    d = _good_desc()
    d["states"] = 17
    with pytest.raises(hb.HeomError) as e:
        hb.Heom(**d)
    assert "heom error -5" in str(e.value)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_loudly():
    with pytest.raises(hb.HeomError) as e:
        hb.Heom(**_good_desc())
    assert "heom error -2" in str(e.value)


def test_ensemble_footprint_groups_classes():
    # host-only: the admission arithmetic needs no device
    t3 = hb.build_tables(hb.System(ho.synthetic_hamiltonian(3, 2), [35] * 3, [50] * 3, [0] * 3, 1, 300.0, 2))
    t3b = dict(t3, hamiltonian=hb.build_tables(hb.System(ho.synthetic_hamiltonian(3, 4), [35] * 3, [50] * 3,
                                                         [0] * 3, 1, 300.0, 2))["hamiltonian"])
    t5 = hb.build_tables(hb.System(ho.synthetic_hamiltonian(5, 2), [35] * 5, [50] * 5, [0] * 5, 2, 300.0, 3))
    one3, one5 = hb.Ensemble.footprint([t3]), hb.Ensemble.footprint([t5])
    # product scheme: state + 2 stage buffers of nodes x sectors x 32 B, plus tables
    assert one5 >= t5["matrices"] * 15 * 32 * 3
    both = hb.Ensemble.footprint([t3, t5])
    assert both == one3 + one5
    # two instances of one class share a handle: states add, and each ADO carries an instance id
    pair = hb.Ensemble.footprint([t3, t3b])
    assert pair > 2 * t3["matrices"] * 5 * 32 * 3 and pair <= 2 * one3 + 4 * 2 * t3["matrices"]
    assert hb.Ensemble.footprint([t3], scheme="reference") > one3


def test_ensemble_footprint_pads_lockstep_classes():
    # 8 or more instances of one class and depth (at most 8 states) form a lockstep class whose
    # state is padded to a multiple of 32 instances; 7 stay a batch; the reference scheme has none
    t = hb.build_tables(hb.System(ho.synthetic_hamiltonian(4, 3), [35] * 4, [50] * 4, [0] * 4, 1, 300.0, 3))
    state1 = int(t["matrices"]) * 8 * 32  # one instance's state: ADOs x 8 pair sectors x 32 B
    seven, eight = hb.Ensemble.footprint([t] * 7), hb.Ensemble.footprint([t] * 8)
    assert eight - seven >= 24 * state1 * 3  # 25 more padded instances, state + 2 stage buffers
    # up to 32 instances the padded state is already counted: only tables and per-instance items grow
    assert hb.Ensemble.footprint([t] * 32) - eight < 24 * state1 * 3
    ref7, ref8 = hb.Ensemble.footprint([t] * 7, scheme="reference"), hb.Ensemble.footprint([t] * 8, scheme="reference")
    assert ref8 - ref7 < 2 * state1 * 6


def test_batch_admission_rejects_mixed_classes():
    t3 = hb.build_tables(hb.System(ho.synthetic_hamiltonian(3, 2), [35] * 3, [50] * 3, [0] * 3, 1, 300.0, 2))
    t3l = hb.build_tables(hb.System(ho.synthetic_hamiltonian(3, 2), [40] * 3, [50] * 3, [0] * 3, 1, 300.0, 2))
    with pytest.raises(hb.HeomError) as e:
        hb.Heom.batch([t3, t3l])
    assert "heom error -1" in str(e.value) and "bath tables differ" in str(e.value)


@pytest.mark.parametrize("m,omega", [(1, 0.0), (2, 0.0), (3, 30.0)])
def test_bath_derivatives_match_central_differences(m, omega):
    # host only: the analytic d(pf_same, pf_circ, cbk)/d(lambda, gamma) against
    # central differences of the tables themselves
    n = 3
    h = ho.synthetic_hamiltonian(n, 4)
    lam, inv = 35.0, 50.0

    def tabs(lam_v, inv_v):
        t = hb.build_tables(hb.System(h, [lam_v] * n, [inv_v] * n, [omega] * n, m, 300.0, 1))
        return np.concatenate([t["pf_same"], t["pf_circ"], t["cbk"]])

    sysd = hb.System(h, [lam] * n, [inv] * n, [omega] * n, m, 300.0, 1)
    for theta in (0, 1):
        ana = np.concatenate(hb.bath_derivatives(sysd, theta))
        if theta == 0:  # per J; lambda in the config is cm^-1
            d = 1e-4 * lam
            fd = (tabs(lam + d, inv) - tabs(lam - d, inv)) / (2 * d * 1.986456217327470903861498336971e-23)
        else:  # per 1/s; gamma = 1 / invnu
            g = 1.0 / (inv * 1e-15)
            d = 1e-5 * g
            fd = (tabs(lam, 1e15 / (g + d)) - tabs(lam, 1e15 / (g - d))) / (2 * d)
        scale = np.max(np.abs(ana))
        assert np.max(np.abs(ana - fd)) <= 1e-7 * scale, (theta, np.max(np.abs(ana - fd)) / scale)


def test_instance_file_round_trip_and_byte_layout(tmp_path):
    """heom_instance_write / read in the reference's binary layout
    (instance.cpp:281-377): fields back to back, native order, no padding."""
    import struct
    sysd = hb.System(ho.synthetic_hamiltonian(3, 6), [35] * 3, [50] * 3, [0] * 3, 2, 300.0, 2)
    t = hb.build_tables(sysd)
    y = np.random.default_rng(0).normal(size=t["matrices"] * 9 * 2)
    path = tmp_path / "inst.bin"
    hb.write_instance(sysd, path, state=y, time=1.25e-13)
    raw = path.read_bytes()
    head = struct.pack("<i?iiidi7q", 0, False, 0, 0, 0, 1.25e-13, t["first_non_plus_id"], 3, t["matrices"], 2, 1,
                       3, 6, 2)
    body = b"".join(np.ascontiguousarray(a).tobytes() for a in (
        y, t["hamiltonian"], t["ado_tuples"], t["ado_plus"], t["ado_minus"], t["pf_same_sum"], t["pf_same"],
        t["pf_circ"], t["cbk"], t["cbk_sqrt"]))
    assert raw == head + body
    tabs, state, tm = hb.read_instance(path)
    assert tm == 1.25e-13 and np.array_equal(state, y)
    for k, v in t.items():
        assert np.array_equal(np.asarray(tabs[k]), np.asarray(v)), k
    # top only: the rest of the state reads back as zeros
    hb.write_instance(sysd, path, state=y[:18], top_only=True)
    _, state, _ = hb.read_instance(path)
    assert np.array_equal(state[:18], y[:18]) and not state[18:].any()


def test_instance_file_rejects_garbage(tmp_path):
    p = tmp_path / "bad.bin"
    p.write_bytes(b"\x07\x00\x00\x00" + b"\x00" * 100)
    with pytest.raises(hb.HeomError) as e:
        hb.read_instance(p)
    assert "heom error -7" in str(e.value)


def test_bench_reports_profiled_traffic_only_for_the_profiled_build(monkeypatch):
    # roofline.traffic comes from the committed ncu summary only when the summary's
    # kernel_source_hash line names the kernel sources being run
    import bench
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles",
                        "heom_dmma_stage_n8_depth8.md")
    recorded = [ln.split("=")[1].strip() for ln in open(path) if ln.startswith("kernel_source_hash")][0]
    monkeypatch.setattr(bench, "kernel_source_hash", lambda: recorded)
    traffic, src = bench.profiled_traffic()
    assert traffic is not None and traffic > 1.5e9 and "this build" in src
    monkeypatch.setattr(bench, "kernel_source_hash", lambda: "0" * 16)
    traffic, src = bench.profiled_traffic()
    assert traffic is None and "another build" in src
