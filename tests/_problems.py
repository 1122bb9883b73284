"""Problem mappings shared by the CPU and GPU tests."""
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import make_golden  # noqa: E402


def golden_problem(name: str) -> dict:
    """The fixture's problem in the provider's JSON mapping form."""
    p = make_golden.template_problem() if name == "template_bgk" else make_golden.channel_problem()
    n = int(np.prod(p["shape"]))
    opts = {"lattice": "D3Q19", "collision": {"kind": p["collision"]}}
    if p.get("box_half_width"):
        opts["filter"] = {"kind": "box", "half_width": p["box_half_width"]}
    out = {k: v for k, v in p.items() if k not in ("collision", "n", "box_half_width")}
    out["history_byte_budget"] = (p["step_count"] + 1) * n * 19 * 8
    out["solver_options"] = opts
    return out


def load_golden(name: str) -> dict:
    d = dict(np.load(Path(__file__).resolve().parent / "golden" / f"{name}.npz"))
    return d
