"""The drop-in with a real caller: the reference's own benchmark driver
main.cc, compiled unchanged (the v8s16 object oracle/Makefile builds from the
reference's sources) and linked against libqws_b200.so in place of the
reference's library (`make -C oracle dropin`; the reference links its main
the same way, Makefile:636-640), run with the arguments of its CASE0 golden
(README:68-80: `./main 32 6 4 3 1 1 1 1 -1 -1 6 50`) on the GPU.

Its output is checked against the reference's data/CASE0 by check.sh's rules
(check.sh:12-31): the same `name : value` / `name^2 = value` lines in the
same order, each within 3e-6 relative for single-precision names, 1e-14 for
the rest, and the final rnorm^2 below 1e-15.  main.cc exercises the
reference-facing C ABI the way a user program does: qws_init_, writing the
glud/glus/clvd/clvs globals and kappa after it, every DD and even-odd
operator it prints a norm of, bicgstab_dd_mix_ and bicgstab_vm_, the norm
helpers, print_timing_ and qws_finalize_.
"""
import json
import os
import subprocess
from pathlib import Path

import pytest

from qwsref import check_sh_ok, parse_golden

ROOT = Path(__file__).resolve().parents[1]
MAIN = ROOT / "oracle" / "_ref" / "main_b200"
GOLD = json.loads((Path(__file__).parent / "golden" / "case_norms.json").read_text())

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not MAIN.exists(),
                                 reason="oracle/_ref/main_b200 not built (make -C oracle dropin)")]


def test_reference_main_linked_against_library_passes_case0():
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "8"))
    res = subprocess.run([str(MAIN), "32", "6", "4", "3", "1", "1", "1", "1", "-1", "-1", "6",
                          "50"], capture_output=True, text=True, env=env, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    got = parse_golden(res.stdout)
    want = GOLD["CASE0"]["norms"]
    assert [k for k, _ in got] == [k for k, _ in want], (got, want)
    bad = [(k, v, r) for (k, v), (_, r) in zip(got, want) if not check_sh_ok(k, v, r)]
    assert not bad, bad
