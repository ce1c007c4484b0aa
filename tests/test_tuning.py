"""CPU: the autotuner's file format (cj_tuning_check_file needs no GPU)."""
import ctypes as C

import pytest

from calamarijoins_b200 import _lib

GOOD = "cj_b200-tuning 1 148\n" + "".join(
    f"class {c} log2_spp {10 + c % 3} part_ctas {2 << (c % 3)} probe_ctas {2 + 2 * (c % 4)}\n" for c in range(6))


def check(path) -> int:
    return _lib.lib().cj_tuning_check_file(str(path).encode())


def test_good_file(tmp_path):
    p = tmp_path / "t.txt"
    p.write_text(GOOD)
    assert check(p) == 0


@pytest.mark.parametrize("bad", [
    "",                                                   # empty
    GOOD.replace("cj_b200-tuning 1", "cj_b200-tuning 2"),  # unknown version
    GOOD.replace("class 5 ", "class 6 "),                 # class out of range (and class 5 missing)
    "\n".join(GOOD.splitlines()[:-1]) + "\n",             # a class missing
    GOOD.replace("log2_spp 11", "log2_spp 15"),            # more slots per partition than shared memory holds
    GOOD.replace("probe_ctas 2", "probe_ctas -1"),         # negative
    GOOD + "garbage\n",                                   # trailing junk
])
def test_malformed_files_rejected(tmp_path, bad):
    p = tmp_path / "t.txt"
    p.write_text(bad)
    assert check(p) == 1  # CJ_ERR_INVALID_ARGUMENT
    assert b"tuning file" in _lib.lib().cj_last_error()


def test_missing_file(tmp_path):
    assert check(tmp_path / "none.txt") == 1
