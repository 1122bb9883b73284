"""The C-ABI without a GPU: the library loads, exports every entry point that
include/lbm_b200.h declares, the header compiles as C99, and lbm_create
rejects invalid problems with the reference's contract messages (the numeric
validation of LbmProblem::normalize, solver.rs:414-550, and normalize_ports,
ports.rs:106-272, runs before any CUDA call)."""
import copy
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from implexity_b200 import ContractError, LbmSolver, _abi, normalize, workloads

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "lbm_b200.h"


def declared():
    return sorted(set(re.findall(r"^LBM_API\s+[\w\s\*]+?\b(lbm_\w+)\s*\(", HEADER.read_text(), re.M)))


def test_every_declared_symbol_is_exported():
    lib = _abi.load()
    names = declared()
    assert len(names) >= 16
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(_abi.EXPORTS) == names
    assert lib.lbm_abi_version() == _abi.ABI_VERSION


def test_header_compiles_as_c99(tmp_path):
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    src = tmp_path / "use.c"
    calls = "\n".join(f"    (void)&{n};" for n in declared())
    src.write_text(f'#include "lbm_b200.h"\nint main(void) {{\n    lbm_problem_t p = {{0}};\n    (void)p;\n{calls}\n    return 0;\n}}\n')
    r = subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), "-c", str(src), "-o",
                        str(tmp_path / "use.o")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError, match="missing"):
        _abi.load(tmp_path / "liblbm_b200.so")


def base():
    return workloads.channel_problem(shape=(10, 8, 6), steps=5, collision="trt")


def expect_contract(problem, message):
    with pytest.raises(ContractError) as e:
        LbmSolver(problem)
    assert message in str(e.value), str(e.value)


def with_(**kw):
    p = base()
    p.update(kw)
    return p


CASES = [
    (dict(kinematic_viscosity_m2_s=1e-9), "Choose spacing/time step such that 0.51 <= relaxation time <= 2"),
    (dict(mach_limit=0.3), "LBM mach_limit must be <= 0.2; this is not a compressible gas solver"),
    (dict(step_count=0), "step_count must be an integer in [1,1000000]"),
    (dict(spacing_m=-1.0), "spacing_m must be a finite positive scalar"),
    (dict(drag_shape=0.0), "drag_shape must be a finite positive scalar"),
    (dict(acceleration_m_s2=[float("nan"), 0, 0]), "acceleration_m_s2 requires three finite components"),
    (dict(history_byte_budget=10), "Population history exceeds explicit byte budget"),
    (dict(shape=[1, 8, 6]), "LBM shape must contain three integers >= 2"),
    (dict(topology_map={"filter_radius_m": 1.0, "projection_beta": 0.0, "projection_eta": 0.5}),
     "filter_radius_m must lie in [0,4*spacing_m]"),
    (dict(topology_map={"filter_radius_m": 0.0, "projection_beta": 40.0, "projection_eta": 0.5}),
     "Require beta in [0,32] and eta in (0,1)"),
    (dict(periodic_axes=[True, False, False]), "A periodic face cannot be a port"),
]


@pytest.mark.parametrize("kw,message", CASES)
def test_contract_messages(kw, message):
    expect_contract(with_(**kw), message)


def test_exact_key_set():
    p = base()
    del p["mach_limit"]
    with pytest.raises(ContractError, match="LBM requires exactly these problem keys"):
        normalize(p)
    p = base()
    p["extra"] = 1
    with pytest.raises(ContractError, match="LBM requires exactly these problem keys"):
        normalize(p)


def test_fixed_design_and_masks():
    p = base()
    p["fixed_design"] = np.full(p["fixed_design"].shape, 1.5)
    expect_contract(p, "fixed_design must be finite and in [0,1]")
    p = base()
    p["solid_mask"] = p["solid_mask"].copy()
    p["solid_mask"][4, 4, 3] = True
    expect_contract(p, "Need fluid cells; fixed solid cells cannot be designable")
    p = base()
    p["solid_mask"] = p["solid_mask"].astype(float)
    expect_contract(p, "solid_mask must be a shape-matched boolean array")


def port_case(mutate, message):
    p = base()
    p["ports"] = copy.deepcopy(p["ports"])
    mutate(p)
    expect_contract(p, message)


def test_port_rules():
    def off_face(p):
        p["ports"][0]["mask"] = p["ports"][0]["mask"].copy()
        p["ports"][0]["mask"][1, 3, 3] = True
    port_case(off_face, "Port mask must lie on its face and cannot overlap another port")

    def edge(p):
        p["ports"][0]["mask"] = p["ports"][0]["mask"].copy()
        p["ports"][0]["mask"][0, 0, 3] = True
    port_case(edge, "Port corners/edges with other closed faces require an unsupported corner closure")

    def designable(p):
        p["design_region"] = p["design_region"].copy()
        p["design_region"][0, 3, 3] = True
    port_case(designable, "Port cells must be protected, unobstructed, fixed-design fluid")

    def normal(p):
        p["ports"][1]["velocity_m_s"] = [1e-6, 0.0, 0.0]
    port_case(normal, "Pressure port velocity specifies tangential components only; normal component must be zero")

    def fast(p):
        p["ports"][0]["velocity_m_s"] = [1.0, 0.0, 0.0]
    port_case(fast, "Authored port velocity exceeds Mach limit")

    def dense(p):
        p["ports"][1]["gauge_pressure_Pa"] = 1e3
    port_case(dense, "Pressure port density must remain within 10% of reference")

    def kind(p):
        p["ports"][0]["kind"] = "mass_flow"
    port_case(kind, "Port kind must be velocity or pressure")

    def dup(p):
        p["ports"][1]["id"] = p["ports"][0]["id"]
    port_case(dup, "Unique port id and exact port fields required")

    def empty(p):
        p["ports"][0]["mask"] = np.zeros_like(p["ports"][0]["mask"])
    port_case(empty, "Nonempty shape-matched boolean port mask required")


def test_collision_parameters():
    p = base()
    p["solver_options"]["collision"] = {"kind": "trt", "magic": -1.0}
    expect_contract(p, "TRT magic parameter must be finite and positive")
    p = base()
    p["solver_options"]["collision"] = {"kind": "mrt", "bulk_rate": 2.5}
    expect_contract(p, "MRT relaxation rates must lie in (0, 2)")
    p = base()
    p["solver_options"]["collision"] = {"kind": "cumulant"}
    with pytest.raises(ContractError, match="collision kind must be bgk, trt or mrt"):
        normalize(p)


def test_ctypes_layouts_match_the_header(tmp_path):
    """Every struct the Python mirrors pass through the C-ABIs (lbm_b200.h,
    mma_cpu.h) has the size and field offsets that the C compiler gives the
    header's declaration."""
    import ctypes as C

    from implexity_b200 import mma

    structs = {"lbm_port_t": _abi.Port, "lbm_problem_t": _abi.Problem, "lbm_diag_t": _abi.Diag,
               "lbm_adjoint_opts_t": _abi.AdjointOpts, "lbm_adjoint_report_t": _abi.AdjointReport,
               "lbm_info_t": _abi.Info, "lbm_slab_diag_t": _abi.SlabDiag, "mma_options_t": mma.Options,
               "mma_info_t": mma.Info, "mma_gcmma_options_t": mma.GcmmaOptions}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "lbm_b200.h"', '#include "mma_cpu.h"',
             "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'    printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    exe = tmp_path / "layout"
    r = subprocess.run([cc, "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


def test_gradient_option_names_are_checked():
    """Unknown option names fail as contract errors before any device call."""
    from implexity_b200.solver import _choice

    assert _choice("mode", "steady", {"horizon": 0, "steady": 1}) == 1
    with pytest.raises(ContractError, match="checkpointing must be one of every, binomial"):
        _choice("checkpointing", "revolve", {"every": 0, "binomial": 1})
