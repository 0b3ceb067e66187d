"""Extract the reference's golden vectors for this path, read as text from its test files and
design document, into reference_pins.json. Run in a container that has the reference checkout:

    python tests/golden/make_reference_pins.py /root/reference

The reference is Julia and does not run here; these are its own tables and recorded numbers.
"""
import json
import re
import sys
from fractions import Fraction
from pathlib import Path


def parse_table(text, name):
    # `const NAME = (k => [a//b, ...], ...)` or `k => [ints] .// den`
    m = re.search(r"const %s = \((.*?)\)\n" % name, text, re.S)
    body = m.group(1)
    out = {}
    for key, arr, den in re.findall(r"(\d+)\s*=>\s*\[([^\]]*)\](?:\s*\.//\s*(\d+))?", body):
        vals = []
        for tok in arr.replace("\n", " ").split(","):
            tok = tok.strip()
            if not tok:
                continue
            if "//" in tok:
                a, b = tok.split("//")
                fr = Fraction(int(a), int(b))
            else:
                fr = Fraction(int(tok))
            if den:
                fr = fr / int(den)
            vals.append([fr.numerator, fr.denominator])
        out[key] = vals
    return out


def main(ref):
    ref = Path(ref)
    st = (ref / "test" / "stencils_tests.jl").read_text()
    code = (ref / "CODE.md").read_text()
    pins = {
        "source": {
            "FD1_TABLE": "test/stencils_tests.jl:41-45",
            "FD2_TABLE": "test/stencils_tests.jl:46-51",
            "KO_TABLE": "test/stencils_tests.jl:54-58",
            "kerr_schild_a0_r1.5": "CODE.md:557-558",
            "box_corner_speed": "CODE.md:977-980",
            "driver_records": "CODE.md:6478-6480",
        },
        "FD1_TABLE": parse_table(st, "FD1_TABLE"),
        "FD2_TABLE": parse_table(st, "FD2_TABLE"),
        "KO_TABLE": parse_table(st, "KO_TABLE"),
    }
    m = re.search(r"so `b = ([0-9.]+)`, `a = ([0-9.]+)` at `r = 1.5 M`", code)
    pins["kerr_schild_a0_r1.5"] = {"b": float(m.group(1)), "a": float(m.group(2)), "M": 1.0, "r": 1.5}
    m = re.search(r"`([0-9.]+)` at half-width `5/2 M`", code)
    pins["box_corner_speed"] = {"lambda": float(m.group(1)), "halfwidth": 2.5, "M": 1.0, "a": 0.0,
                                "digits": len(m.group(1).split(".")[1])}
    m = re.search(r"hole's `err_l2 =\s+([0-9.]+)e.([0-9]+)`.*?wave's is\s+`([0-9.]+)e.([0-9]+)`", code, re.S)
    pins["driver_records"] = {"hole_fixture_err_l2": float(m.group(1)) * 10.0 ** -int(m.group(2)),
                              "gauge_wave_err_l2": float(m.group(3)) * 10.0 ** -int(m.group(4)),
                              "gauge_wave_setup": "bench/stepping.jl:73-82,160-181: gauge_wave_case(eps_KO=1/2, "
                                                  "gamma0=1, gamma2=0), N=16, roots=8, q=4, chunk=1/50, t_end=3/50"}
    Path(__file__).with_name("reference_pins.json").write_text(json.dumps(pins, indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
