"""Extract the reference's golden norms into a JSON fixture.

Reads the reference's own golden outputs data/CASE* (produced by its main
driver, README:68-80) with check.sh's extraction rule (`name : value` and
`name^2 = value` lines, check.sh:12-14) and records, per case, the command
arguments (local lattice, rank grid) next to the list of (name, value).

Run in a container that has the reference checked out:
    python tests/golden/make_golden.py $QWS_REFERENCE/data > tests/golden/case_norms.json
"""
import json
import os
import re
import sys
from pathlib import Path

# README:68-80: ./main lx ly lz lt px py pz pt tol tol_s maxiter+1 maxiter_s
CASES = {
    "CASE0": ((32, 6, 4, 3), (1, 1, 1, 1), {"vlend": 8, "vlens": 16}),
    "CASE1": ((32, 6, 4, 3), (1, 1, 1, 2), {"vlend": 8, "vlens": 16}),
    "CASE2": ((32, 3, 4, 4), (1, 1, 1, 2), {"vlend": 8, "vlens": 16}),
    "CASE3": ((32, 3, 6, 4), (1, 1, 1, 2), {"vlend": 8, "vlens": 16}),
    "CASE4": ((32, 6, 6, 2), (1, 1, 1, 2), {"vlend": 8, "vlens": 16}),
    "CASE5": ((32, 6, 6, 4), (1, 1, 1, 2), {"vlend": 8, "vlens": 16}),
    "CASE6": ((32, 6, 6, 8), (1, 1, 1, 2), {"vlend": 8, "vlens": 16}),
    "CASE7": ((32, 6, 4, 3), (1, 2, 2, 2), {"vlend": 8, "vlens": 16}),
    "CASE8": ((32, 6, 4, 3), (4, 4, 1, 1), {"vlend": 8, "vlens": 16}),
    "CASE9": ((32, 6, 4, 3), (1, 1, 4, 4), {"vlend": 8, "vlens": 16}),
    "CASE_4111_1111": ((4, 1, 1, 1), (1, 1, 1, 1), {"vlend": 2, "vlens": 2}),
    "CASE_4111_1111_HP": ((4, 1, 1, 1), (1, 1, 1, 1), {"vlend": 2, "vlens": 2, "half_prec": 1}),
}


def extract(text):
    out = []
    for line in text.splitlines():
        if "git commit hash" in line:
            continue
        if re.search(r" : +[0-9]|2 += +[0-9]", line):
            parts = line.split()
            out.append([parts[0], float(parts[-1])])
    return out


def extract_hp_history(text):
    """The half-precision golden's residual history lines (@D outer,
    @C true inner, @@ recursive inner), in order."""
    hist = []
    for line in text.splitlines():
        m = re.match(r"^(@D|@C|@@)\s+(\d+)\s+(\S+)", line)
        if m:
            hist.append([m.group(1), int(m.group(2)), float(m.group(3))])
    return hist


def main():
    data = Path(sys.argv[1] if len(sys.argv) > 1 else
                os.path.join(os.environ.get("QWS_REFERENCE", "/root/reference"), "data"))
    res = {}
    for name, (lloc, npe, opts) in CASES.items():
        text = (data / name).read_text()
        entry = {"lloc": lloc, "npe": npe, "args": {"tol": -1, "tol_s": -1, "maxiter": 6,
                                                    "maxiter_s": 50, "nsap": 4, "nm": 2,
                                                    "kappa": 0.05, "fbc": [1, 1, 1, -1]},
                 "norms": extract(text)}
        entry.update(opts)
        if opts.get("half_prec"):
            entry["hp_history"] = extract_hp_history(text)
        res[name] = entry
    json.dump(res, sys.stdout, indent=1)
    sys.stdout.write("\n")


if __name__ == "__main__":
    main()
