"""Writes tests/golden/quicktest_uniform.json from the flowPsi reference's own
quick tests (quickTest/inviscid/{inflow,isentropic,fixedMass,superSonic}.{vars,dat,tol.dat}).

Each of these four tests drives a duct of unit cross-section from an
inflow condition to an outflow condition and extracts P, T and u at every
node after it has converged; every node holds the same uniform state, which
therefore depends only on the two boundary conditions, not on the grid
(`testGrid.vog`, which is not read here).  The script records, per test, the
boundary options, the initial state, the pseudo-time step settings, the
expected uniform state and the test's tolerances.

    python tests/golden/make_quicktest_uniform.py /path/to/flowPsi
"""
import json
import re
import sys
from pathlib import Path

TESTS = ("inflow", "isentropic", "fixedMass", "superSonic")


def number(text: str, key: str) -> float:
    m = re.search(r"\b" + key + r"\s*=\s*([-+0-9.eE]+)", text)
    if not m:
        raise ValueError(f"no {key}= in {text!r}")
    return float(m.group(1))


def parse(ref: Path, name: str) -> dict:
    d = ref / "quickTest" / "inviscid"
    src = (d / f"{name}.vars").read_text()
    vars_ = re.sub(r"//[^\n]*", "", src)  # drop comments
    bcs = dict(re.findall(r"(BC_\d+)\s*=\s*([A-Za-z]+\([^)]*\)|[A-Za-z]+)", vars_))
    inflow = bcs["BC_5"]
    outflow = bcs["BC_6"]
    kind = inflow.split("(")[0]
    opts = inflow[len(kind):]
    bc = {"kind": kind}
    if kind in ("inflow", "supersonicInflow"):
        bc.update(p=number(opts, "p"), T=number(opts, "T"), u=number(opts, "u"))
    elif kind == "isentropicInflow":
        bc.update(p0=number(opts, "p0"), T0=number(opts, "T0"))
    elif kind == "fixedMass":
        bc.update(mdot=number(opts, "mdot"), T0=number(opts, "T0"))
    else:
        raise ValueError(kind)
    assert outflow.startswith("outflow(") or outflow == "supersonicOutflow"
    ic = re.search(r"initialConditions\s*:\s*<([^>]*)>", vars_).group(1)
    init = {"p": number(ic, "p"), "T": number(ic, "T")}
    if re.search(r"\bu\s*=", ic):
        init["u"] = number(ic, "u")
    else:
        init["M"] = number(ic, "M")
    rows = {tuple(line.split()) for line in (d / f"{name}.dat").read_text().splitlines() if line.strip()}
    assert len(rows) == 1, f"{name}.dat is not uniform"
    P, T, u = (float(v) for v in rows.pop())
    tol = [float(v) for v in (d / f"{name}.tol.dat").read_text().split()]
    return {"inflow": bc, "init": init,
            "outflow": {"kind": "supersonicOutflow"} if outflow == "supersonicOutflow" else
                       {"kind": "outflow", "p": number(outflow, "p")},
            "regime": re.search(r"flowRegime\s*:\s*(\w+)", vars_).group(1),
            "dtmax": number(vars_.replace(":", "="), "dtmax"),
            "urelax": number(vars_.replace(":", "="), "urelax"),
            "stop_iter": int(number(vars_.replace(":", "="), "stop_iter")),
            "expect": {"P": P, "T": T, "u": u}, "tol": tol,
            "source": f"quickTest/inviscid/{name}.vars, .dat, .tol.dat"}


def main(ref: str) -> None:
    out = {name: parse(Path(ref), name) for name in TESTS}
    dst = Path(__file__).resolve().parent / "quicktest_uniform.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
