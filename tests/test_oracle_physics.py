"""The reference's analytic known-answer tests on the oracle (CPU): pins the restatement of CpuSolver."""
import pytest

from physics_cases import CASES


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_known_answers(oracle_mod, case):
    CASES[case](lambda: oracle_mod.OracleSolver())
