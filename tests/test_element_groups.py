"""Material groups of an input deck (setElementMaterial block of
BasicModel::ProcessSetElementProperty, BasicModel.cpp:682-775): the C ABI
parser against known answers and the oracle restatement; malformed or
undefined input is refused."""
import numpy as np
import pytest

from betanoox_b200 import BetaGpuError, _abi, parse_element_groups

BLOCK = """// material groups
0 9 1 2
10 19 2 5      // every other element
/* a comment
   over lines */ 11 19 2 7
end
0 19 1 9
"""


def test_known_block(oracle):
    g = parse_element_groups(BLOCK, 20)
    want = [2] * 10 + [5, 7] * 5
    assert g.tolist() == want
    assert oracle.element_groups_from_block(BLOCK, 20) == want


def test_all_then_ranges_and_terminators(oracle):
    text = "all 1\n3 6 3 4\n-1\n0 0 1 8\n"
    assert parse_element_groups(text, 8).tolist() == [1, 1, 1, 4, 1, 1, 4, 1]
    assert parse_element_groups("ALL 3\nEnd\n0 1 1 2", 3).tolist() == [3, 3, 3]
    assert parse_element_groups("2 2 1 6", 4, init=0).tolist() == [0, 0, 6, 0]


def test_random_blocks_match_oracle(oracle):
    rng = np.random.default_rng(4)
    for _ in range(50):
        n = int(rng.integers(5, 200))
        lines = []
        for _ in range(int(rng.integers(1, 8))):
            if rng.random() < 0.15:
                lines.append(f"all {int(rng.integers(0, 9))}")
            else:
                a = int(rng.integers(0, n))
                b = int(rng.integers(a, n))
                lines.append(f"{a}\t{b} {int(rng.integers(1, 5))} {int(rng.integers(0, 9))}")
        text = "\n".join(lines) + "\nend\n"
        assert parse_element_groups(text, n).tolist() == oracle.element_groups_from_block(text, n)


@pytest.mark.parametrize("text", ["0 5 1\n", "0 20 1 2\n", "0 5 0 1\n", "6 5 1 1\n", "0 5 1 x\n",
                                  "all\n", "0 5 1 -2\n", "/* open\n0 1 1 1\n"])
def test_refused(oracle, text):
    with pytest.raises(BetaGpuError) as e:
        parse_element_groups(text, 20)
    assert e.value.status == _abi.ERR_ARG
    assert oracle.element_groups_from_block(text, 20) is None
