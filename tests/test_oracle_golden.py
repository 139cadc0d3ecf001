"""The oracle against the reference's own golden values
(examples/plugins/notebooks/01_c_plugins.ipynb, 02_rust_plugins.ipynb),
through tests/golden/plugin_notebooks.json."""

import math

import numpy as np
import pytest
from harness import golden_fixture, golden_problem, run_oracle
from oracle_client import REF_PLUGINS

CASES = golden_fixture()["cases"]
BUILTIN = [c for c in CASES if "plugin" not in c]
PLUGIN = [c for c in CASES if "plugin" in c]


def _problem(case):
    p = golden_problem()
    p.max_weight = case.get("max_weight")
    p.min_coeff = case.get("min_coeff")
    if "noise" in case:
        d = case["noise"]["uniform"]
        p.noise_table = np.array([math.exp(-d * float(w)) for w in range(p.n_units + 1)])
    return p


@pytest.mark.parametrize("case", BUILTIN, ids=[c["name"] for c in BUILTIN])
def test_builtin_golden_values_bit_exact(oracle, case):
    # The notebook ran with n_threads=4; the built-in cases are bit-exact here.
    r = run_oracle(oracle, _problem(case), n_partitions=4)
    assert r.expectation == case["expected"]


@pytest.mark.parametrize("case", PLUGIN, ids=[c["name"] for c in PLUGIN])
def test_plugin_golden_values(oracle, case):
    so = REF_PLUGINS / f"{case['plugin']}.so"
    if not so.exists():
        pytest.skip("reference example plugins not built (oracle/build_ref_plugins.sh)")
    h = oracle.load_plugin(so, case["plugin_config"], noise=case["plugin_kind"] == "noise")
    try:
        p = golden_problem()
        kw = {"noise_plugin": h} if case["plugin_kind"] == "noise" else {"truncator": h}
        r = oracle.run(p.basis, p.n_units, p.n_words, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets,
                       diag_state=p.diag, n_partitions=4, **kw)
    finally:
        oracle.lib.pqo_plugin_free(h)
    # Partition-sum order differs from FxHash partitioning: allow the last bits.
    assert abs(r.expectation - case["expected"]) <= 1e-12 * abs(case["expected"])


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_partition_count_does_not_change_terms(oracle, parts):
    # crates/core/tests/unit/engine/partitioned_termsum.rs: identical results for every partition count.
    p = golden_problem(min_coeff=1e-3)
    base = run_oracle(oracle, p, n_partitions=1)
    r = run_oracle(oracle, p, n_partitions=parts)
    ka = {tuple(k): c for k, c in zip(base.keys.tolist(), base.coeffs.tolist())}
    kb = {tuple(k): c for k, c in zip(r.keys.tolist(), r.coeffs.tolist())}
    assert ka == kb
    assert np.array_equal(base.n_terms, r.n_terms)
