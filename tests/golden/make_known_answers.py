"""Extract the known-answer tests of Zinq's quantum-dynamics path into a JSON fixture.

Source: test/quantum_dynamics.zig:8-282 of tjira/zinq (ten end-to-end tests,
tolerance TEST_TOLERANCE = 1e-8 at :6).  The script reads that Zig file as
text, turns each ``Options{...}`` literal into the reference JSON schema
(src/quantum_dynamics.zig:25-67) and records the expected final observables.

Usage (in a checkout that has the reference tree):
    python tests/golden/make_known_answers.py <zinq-root> > tests/golden/known_answers.json
"""
from __future__ import annotations

import json
import re
import sys


def _nums(s):
    return [float(x) for x in re.findall(r"-?\d+(?:\.\d+)?(?:e-?\d+)?", s)]


def parse(path):
    text = open(path).read()
    tol = float(re.search(r"TEST_TOLERANCE\s*=\s*([0-9.e-]+)", text).group(1))
    tests = []
    for m in re.finditer(r'test "([^"]+)" \{(.*?)\n\}', text, re.S):
        name, body = m.group(1), m.group(2)
        line = text[: m.start()].count("\n") + 1
        opt = {}
        g = re.search(r"\.grid = \.\{ \.bounds = &\.\{(.*?)\}, \.npoint = (\d+) \}", body)
        bounds = [_nums(b) for b in re.findall(r"\.\{([^{}]*)\}", g.group(1))]
        opt["grid"] = {"bounds": bounds, "npoint": int(g.group(2))}
        ic = re.search(r"\.initial_conditions = \.\{(.*?)\},\n", body).group(1)
        icd = {}
        for key in ("momentum", "position", "gamma"):
            icd[key] = _nums(re.search(r"\." + key + r" = &\.\{([^}]*)\}", ic).group(1))
        st = re.search(r"\.state = (\d+)", ic)
        if st:
            icd["state"] = int(st.group(1))
        ad = re.search(r"\.adiabatic = (true|false)", ic)
        if ad:
            icd["adiabatic"] = ad.group(1) == "true"
        opt["initial_conditions"] = icd
        pot = re.search(r"\.potential = \.\{ \.(\w+) = \.\{(.*?)\} \},\n", body)
        pargs = {}
        km = re.search(r"\.k = &\.\{([^}]*)\}", pot.group(2))
        if km:
            pargs["k"] = _nums(km.group(1))
        opt["potential"] = {pot.group(1): pargs}
        im = re.search(r"\.imaginary = \.\{ \.nstate = (\d+) \}", body)
        if im:
            opt["imaginary"] = {"nstate": int(im.group(1))}
        opt["fft"] = {"plan": re.search(r"\.fft = \.\{ \.plan = \.(\w+) \}", body).group(1)}
        opt["mass"] = _nums(re.search(r"\.mass = &\.\{([^}]*)\}", body).group(1))
        opt["iterations"] = int(re.search(r"\.iterations = (\d+)", body).group(1))
        opt["time_step"] = _nums(re.search(r"\.time_step = ([0-9.e-]+)", body).group(1))[0]
        top_ad = re.search(r"\n\s+\.adiabatic = (true|false),", body)
        if top_ad:
            opt["adiabatic"] = top_ad.group(1) == "true"
        expect = []
        for em in re.finditer(r"items\[(\d+)\]\.(\w+)\.\?(?:\.at\((\d+)\))?,\s*(-?[0-9.]+), TEST_TOLERANCE", body):
            expect.append({"solve": int(em.group(1)), "field": em.group(2),
                           "index": None if em.group(3) is None else int(em.group(3)),
                           "value": float(em.group(4)), "text": em.group(4)})
        tests.append({"name": name, "source": f"test/quantum_dynamics.zig:{line}", "options": opt, "expect": expect})
    return {"tolerance": tol, "tests": tests}


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else "."
    print(json.dumps(parse(root + "/test/quantum_dynamics.zig"), indent=1))
