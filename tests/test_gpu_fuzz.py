"""The CUDA flavor against the oracle on the seeded random plans of
tests/test_oracle_reference_fuzz.py (where the oracle itself is checked against the reference on
the same plans and data): selections, projections, hash / global / emitting roots and Join01
probe chains, default flavor, bit-exact."""
import pytest

from oracle.voila_oracle import result_lines, run_plan
from test_oracle_reference_fuzz import SPEC, STAR_SPEC, random_join_plan, random_plan
from vldb_voila_b200 import Engine, generate_workload_host, workload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spec,make,seeds", [(SPEC, random_plan, range(1000, 1008)),
                                             (STAR_SPEC, random_join_plan, range(2000, 2006))],
                         ids=["single_table", "join_chains"])
def test_random_plans_match_oracle(spec, make, seeds):
    w = workload(spec)
    data = generate_workload_host(w)
    e = Engine(0)
    e.load_workload(w, data=data)
    for seed in seeds:
        plan = make(seed)
        q = e.query(plan)
        q.run()
        assert q.result_lines() == result_lines(run_plan(plan, data)), plan
        q.close()
    e.close()
