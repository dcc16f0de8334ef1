"""nim_exp, the exp of the device NIM coefficients, restates glibc's exp
(Arm optimized-routines' table-driven algorithm, FMA build) and must equal
the host libm's exp bit for bit: the exponential form of the NIM constants
(nim.f90:190-194, 375-379) amplifies one ulp of exp near |Pe| = v_limit by
~1e7, so any other exp would move the GPU path away from the reference's
arithmetic.  Here, on the CPU: the table against 2^(j/128) recomputed in
80-digit decimal arithmetic, and the host build of the same source against
libm over 6e7 arguments."""
import re
import sys
from pathlib import Path

import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent))
import _exp_harness as H  # noqa: E402

CSRC = H.CSRC
sys.path.insert(0, str(CSRC))
import gen_exp_table  # noqa: E402


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    return H.build(tmp_path_factory.mktemp("exp"))


def test_table_is_two_to_the_j_over_128():
    text = (CSRC / "nim_exp.cuh").read_text()
    block = text.split("#define NIM_EXP_TABLE_INIT {", 1)[1].split("}", 1)[0]
    got = [int(v, 16) for v in re.findall(r"0x([0-9a-f]{16})ULL", block)]
    assert got == gen_exp_table.entries()


@pytest.mark.parametrize("kind,lo,hi,n", [
    (0, 1e-2, 50.0, 20_000_000),     # the cell Peclet numbers of the exponential branch
    (0, 1e-20, 745.0, 10_000_000),   # tiny to overflow / subnormal results
    (0, 500.0, 745.0, 10_000_000),   # the two-factor scaling range
    (1, 0.0, 0.0, 20_000_000),       # every double, NaN and inf included
])
def test_host_build_matches_libm(harness, kind, lo, hi, n):
    assert harness.count_mismatch(n, 20241204 + kind, kind, lo if lo else 1.0, hi if hi else 2.0) == 0
