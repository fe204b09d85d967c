"""The particle sources' counter-based generator (Philox-4x32-10, Salmon et
al., SC'11), called through the C ABI on the host: the published known-answer
vectors of the algorithm's reference implementation (Random123 kat_vectors,
philox4x32 with 10 rounds)."""
import numpy as np
import pytest

from rhybrid_b200 import abi

KAT = [
    ([0x00000000, 0x00000000, 0x00000000, 0x00000000], [0x00000000, 0x00000000],
     [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff, 0xffffffff, 0xffffffff, 0xffffffff], [0xffffffff, 0xffffffff],
     [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
]


@pytest.mark.parametrize("ctr,key,expected", KAT)
def test_philox_known_answers(ctr, key, expected):
    assert abi.philox4x32(abi.gpu_library(), ctr, key) == expected


def test_philox_words_are_uniform():
    """Counter increments give uniform, uncorrelated words (a coarse check)."""
    lib = abi.gpu_library()
    w = np.array([abi.philox4x32(lib, [i, 7, 0, 1], [12345, 678]) for i in range(4096)], dtype=np.float64)
    u = w / 2.0 ** 32
    assert abs(u.mean() - 0.5) < 0.01
    assert abs(u.var() - 1.0 / 12.0) < 0.003
    assert abs(np.corrcoef(u[:-1, 0], u[1:, 0])[0, 1]) < 0.05
