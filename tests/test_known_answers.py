"""The reference's known-answer tests (delays, queues, multiple runs, the example run),
checked on the CPU oracle (pins the oracle) and on the CUDA library (parity)."""
import pytest

import _cases

IDS = [c.__name__ for c in _cases.ALL]


@pytest.mark.parametrize("case", _cases.ALL, ids=IDS)
def test_oracle_known_answer(case, oracle_factory):
    case(oracle_factory)


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases.ALL, ids=IDS)
def test_gpu_known_answer(case, gpu_factory):
    case(gpu_factory)
