"""Comparison of bra's printed output (shared by the .qcx tests).

Printed numbers are compared to within one unit of the last printed digit
(bra prints 3 to 9 digits; a value at a rounding boundary or a signed zero may
print differently); integers (indices, bit strings, outcomes) exactly; other
text exactly.  Timing lines ("... finished: t (dt)") are dropped first."""
import re

NUM = re.compile(r"^[-+]?(\d+\.?\d*|\.\d+)([eE][-+]?\d+)?$")
INT = re.compile(r"^[-+]?\d+$")
TIMING = re.compile(r"finished: [-+0-9.eE]+ \([-+0-9.eE]+\)$")


def without_timings(text):
    return "\n".join(line for line in text.splitlines() if not TIMING.search(line))


def last_digit(tok):
    """Unit in the last printed digit of a decimal token."""
    mant, _, exp = tok.lower().partition("e")
    decimals = len(mant.split(".")[1]) if "." in mant else 0
    return 10.0 ** (-decimals + (int(exp) if exp else 0))


def same_output(got, want):
    gl, wl = got.splitlines(), want.splitlines()
    assert len(gl) == len(wl), (got, want)
    for g, w in zip(gl, wl):
        gt = re.split(r"([\s(),]+)", g)
        wt = re.split(r"([\s(),]+)", w)
        assert len(gt) == len(wt), (g, w)
        for a, b in zip(gt, wt):
            if NUM.match(b) and NUM.match(a):
                a_int, b_int = INT.match(a), INT.match(b)
                if a_int and b_int:  # integers (indices, bit strings, outcomes, a zero): equal values
                    assert (a == b) if len(b) > 1 and set(b) <= {"0", "1"} else float(a) == float(b), (g, w)
                else:  # a value printed as an integer on one side (a zero) takes the other side's digits
                    unit = last_digit(a) if b_int else last_digit(b)
                    assert abs(float(a) - float(b)) <= max(1e-12, 1.01 * unit), (g, w)
            elif a.strip() != b.strip():
                assert a == b, (g, w)
