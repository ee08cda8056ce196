"""The launch order of live slots (csrc/kr_order.h): template ascending, then
remaining steps descending, ties in slot-list order -- compiled with g++ on
the host and compared with Python's stable sort on the same key, including
the cases whose digits are all equal (one template, short horizons) and the
largest remaining-step counts."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "kraken_3_gpu_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "kr_order.h"
int main() {
  int n;
  if (scanf("%d", &n) != 1) return 1;
  std::vector<int> tpl(n), rem(n), perm, perm2;
  std::vector<uint64_t> k1, k2;
  for (int i = 0; i < n; i++)
    if (scanf("%d %d", &tpl[i], &rem[i]) != 2) return 1;
  krb::lpt_order(n, tpl.data(), rem.data(), perm, k1, k2, perm2);
  for (int i = 0; i < n; i++) printf("%d\n", perm[i]);
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    d = tmp_path_factory.mktemp("order")
    src = d / "order.cpp"
    src.write_text(DRIVER)
    exe = d / "order"
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", CSRC, str(src), "-o", str(exe)],
                   check=True)
    return str(exe)


def run(driver, tpl, rem):
    inp = f"{len(tpl)}\n" + "".join(f"{t} {r}\n" for t, r in zip(tpl, rem))
    out = subprocess.run([driver], input=inp, capture_output=True, text=True, check=True).stdout
    return [int(x) for x in out.split()]


def expected(tpl, rem):
    return sorted(range(len(tpl)), key=lambda i: (tpl[i], -rem[i], i))


CASES = {
    "empty": ([], []),
    "one": ([3], [17]),
    "one_template_short": (None, (1, 4097)),        # digit 0 and part of digit 1 vary
    "many_templates": (72, (1, 4097)),
    "long_horizons": (8, (1, 1 << 30)),
    "max_values": (None, None),
    "all_equal": (None, (5, 6)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_lpt_order_matches_stable_sort(driver, name):
    rng = np.random.default_rng(sum(name.encode()))
    spec = CASES[name]
    if name == "max_values":
        tpl = [255, 0, 255, 0, 7] * 40
        rem = [2**31 - 1, 2**31 - 1, 0, 0, 2**30] * 40
    elif isinstance(spec[0], list):
        tpl, rem = spec
    else:
        n = 5000
        n_tpl = spec[0] or 1
        tpl = rng.integers(0, n_tpl, n).tolist()
        rem = rng.integers(spec[1][0], spec[1][1], n).tolist()
    got = run(driver, tpl, rem)
    assert got == expected(tpl, rem)
