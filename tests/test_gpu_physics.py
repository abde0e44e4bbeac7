"""The reference's analytic known-answer tests on the CUDA solver, through the C ABI."""
import pytest

from physics_cases import CASES


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_cuda_known_answers(gpu, case):
    CASES[case](lambda: gpu.CudaSolver(0))
