"""Regenerates tests/golden/plugin_notebooks.json from the reference tree.

The reference's plugin notebooks (examples/plugins/notebooks/01_c_plugins.ipynb,
cells 4-6, and 02_rust_plugins.ipynb, cells 4 and 8) run a 4-qubit circuit of
40 rotations drawn with Python's random.seed(0), observable Z_0, initial state
0 and n_threads=4, and print the expectation value for built-in and plugin
noise / truncation.  This script rebuilds that circuit exactly as the notebook
does and reads the printed values out of the stored notebook outputs, so the
fixture carries both the inputs and the reference's own answers.

Run from the repository root:  python tests/golden/make_golden.py <reference tree>
(or with the tree in the PROPAQ_REFERENCE environment variable).
"""

import json
import random
import re
import sys
from pathlib import Path

import os

if len(sys.argv) < 2 and not os.environ.get("PROPAQ_REFERENCE"):
    sys.exit("usage: make_golden.py <reference tree>  (or set PROPAQ_REFERENCE)")
REF = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ["PROPAQ_REFERENCE"])
NB = REF / "examples" / "plugins" / "notebooks"
OUT = Path(__file__).resolve().parent / "plugin_notebooks.json"
N_QUBITS = 4


def circuit():
    """random_circuit(depth=40) of the notebooks: PauliString(x, z, 4), angle U[0.05, 0.6)."""
    random.seed(0)
    rots = []
    for _ in range(40):
        x = random.randint(0, 2**N_QUBITS - 1)
        z = random.randint(0, 2**N_QUBITS - 1)
        if x == 0 and z == 0:
            x = 1
        rots.append({"x": x, "z": z, "angle": random.uniform(0.05, 0.6)})
    return rots


def outputs(nb_path):
    nb = json.loads(nb_path.read_text())
    text = []
    for cell in nb["cells"]:
        for o in cell.get("outputs", []):
            if "text" in o:
                text.append("".join(o["text"]))
    return "\n".join(text)


def main():
    out1 = outputs(NB / "01_c_plugins.ipynb")
    out2 = outputs(NB / "02_rust_plugins.ipynb")
    cases = []
    m = re.search(r"uniform_noise:\s+native=(\S+) built-in=(\S+)", out1)
    cases.append({"name": "uniform_noise_builtin", "noise": {"uniform": 0.01}, "expected": float(m.group(2)),
                  "source": "examples/plugins/notebooks/01_c_plugins.ipynb cell 6"})
    m = re.search(r"weight_truncator:\s+native=(\S+) built-in=(\S+)", out1)
    cases.append({"name": "weight_truncator_builtin", "max_weight": 3, "expected": float(m.group(2)),
                  "source": "examples/plugins/notebooks/01_c_plugins.ipynb cell 6"})
    m = re.search(r"pareto\(alpha=0\):\s+native=(\S+) built-in=(\S+)", out1)
    cases.append({"name": "coefficient_truncator_builtin", "min_coeff": 1e-3, "expected": float(m.group(2)),
                  "source": "examples/plugins/notebooks/01_c_plugins.ipynb cell 6"})
    configs = {
        "uniform_noise": ('{"damping": 0.01}', "noise"),
        "thermal_decay_noise": ('{"gamma": 0.02, "beta": 1.6}', "noise"),
        "drifting_noise": ('{"damping": 0.01, "drift_rate": 0.0001}', "noise"),
        "depth_dependent_noise": ('{"damping": 0.02, "rate": 3.0}', "noise"),
        "qubit_local_noise": ('{"damping": 0.05, "mask": 5}', "noise"),
        "weight_truncator": ('{"max_weight": 3}', "trunc"),
        "pareto_truncator": ('{"threshold": 1e-2, "alpha": 2.0}', "trunc"),
        "stochastic_truncator": ('{"threshold": 0.3, "seed": 11}', "trunc"),
        "support_truncator": ('{"threshold": 1e-3, "alpha": 1.0, "mask": 3}', "trunc"),
    }
    for name, (cfg, kind) in configs.items():
        m = re.search(rf"^{name}\s+C=(\S+)\s+Rust=(\S+)", out2, re.M)
        cases.append({"name": f"plugin_{name}", "plugin": name, "plugin_kind": kind, "plugin_config": cfg,
                      "expected": float(m.group(1)),
                      "source": "examples/plugins/notebooks/02_rust_plugins.ipynb cell 8"})
    fixture = {"n_qubits": N_QUBITS, "observable": {"x": 0, "z": 1, "coeff": 1.0}, "initial_state": 0,
               "n_threads": 4, "layers": "one rotation per layer (PauliCircuit of a flat list)",
               "rotations": circuit(), "cases": cases}
    OUT.write_text(json.dumps(fixture, indent=1))
    print(f"wrote {OUT} with {len(cases)} cases")


if __name__ == "__main__":
    main()
