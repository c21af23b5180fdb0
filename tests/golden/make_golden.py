"""Generate the golden residue fixtures under tests/golden/.

Run from the repository root:  python tests/golden/make_golden.py <set> [...]

Sets:
  small  residues of small exponents from the independent big-integer model
         (oracle/bigint_model.py), several lengths, LL and PRP
  c1     full Lucas-Lehmer tests of q = 44497 (a Mersenne prime exponent) and
         the next 8 primes, at n = 2048 (the reference's length) and 4096,
         from the C oracle
  c2     q = 139000003 (first prime above 1.39e8) at n = 2^23: Res64 after 1000
         iterations (and 10000 with --c2-long) from the C oracle
  ref    parse the reference build's residue dumps collected on a B200
         (gpurun_out/ref_*/) into ref_residues.json

Every fixture records how it was made.  The oracle and the model are test
infrastructure; see oracle/lnt_oracle.c for what they restate.
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import bigint_model as B  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = Path(__file__).resolve().parent

C1_EXPONENTS = [44497, 44501, 44507, 44519, 44531, 44533, 44537, 44543, 44549]
C2_EXPONENT = 139000003


def is_prime(k: int) -> bool:
    if k < 2:
        return False
    i = 2
    while i * i <= k:
        if k % i == 0:
            return False
        i += 1
    return True


def write(name: str, obj) -> None:
    (HERE / name).write_text(json.dumps(obj, indent=1) + "\n")
    print("wrote", HERE / name)


def make_small() -> None:
    cases = []
    exps = [89, 101, 127, 257, 521, 607, 1009, 1279, 2203, 3217, 4099, 4253, 9689, 9973, 11213]
    for q in exps:
        n0 = 1 << O.secured_log2(q)
        for n in sorted({n0, 2 * n0}):
            if n > q or -(-q // n) > 30:
                continue
            for prp in (False, True):
                for k in (1, 2, 10, 100):
                    v = B.run(q, k, prp)
                    cases.append({"q": q, "n": n, "prp": prp, "iterations": k,
                                  "res64": f"{B.res64(v):016x}",
                                  "digits_head": [int(d) for d in B.to_digits(v, q, n)[:4]]})
    write("small_bigint.json", {
        "source": "oracle/bigint_model.py (exact big-integer model of r2b/m2 semantics)",
        "cases": cases})


def make_c1() -> None:
    O.set_threads(O.max_threads())
    out = []
    for q in C1_EXPONENTS:
        for n in (2048, 4096):
            t0 = time.time()
            with O.OracleTest(q, n, prp=False) as T:
                T.iterate(q - 2)
                out.append({"q": q, "n": n, "prp": False, "iterations": q - 2,
                            "res64": f"{T.res64():016x}", "is_prime": T.is_prime()})
            print(q, n, out[-1]["res64"], out[-1]["is_prime"], f"{time.time() - t0:.1f}s", flush=True)
    write("c1_oracle.json", {"source": "oracle/lnt_oracle.c, full LL from s0 = 4", "cases": out})


def make_c2(long_run: bool) -> None:
    O.set_threads(O.max_threads())
    marks = [1, 2, 10, 100, 1000] + ([10000] if long_run else [])
    res = {}
    with O.OracleTest(C2_EXPONENT, 1 << 23, prp=False) as T:
        done = 0
        t0 = time.time()
        for m in marks:
            T.iterate(m - done)
            done = m
            res[str(m)] = f"{T.res64():016x}"
            print(m, res[str(m)], f"{time.time() - t0:.0f}s", flush=True)
    name = "c2_oracle_long.json" if long_run else "c2_oracle.json"
    write(name, {"source": "oracle/lnt_oracle.c, LL from s0 = 4", "q": C2_EXPONENT,
                 "n": 1 << 23, "res64_after": res})


def make_ref() -> None:
    """Collect the reference runs summarised by oracle/run_ref.py on a B200
    (gpurun_out/ref_*/run_*.json: Res64 of its LucasNTT_results.dat dump)."""
    base = ROOT / "gpurun_out"
    cases = []
    for js in sorted(base.glob("ref_*/run_*.json")):
        r = json.loads(js.read_text())
        if r.get("rc") != 0 or not r.get("res64"):
            continue
        cases.append({"q": r["exponent"], "n": r["n"], "prp": r["prp"], "iterations": r["iterations"],
                      "res64": r["res64"], "fft": r["fft_used"], "pool": r["pool"],
                      "per_iteration_ms": r["per_iteration_ms"], "conclusion": r["conclusion"],
                      "dump_sha256": r.get("sha256_of_dump")})
    write("ref_residues.json", {
        "source": "reference LucasNTT build (oracle/build_ref.sh) run on a B200 by oracle/run_ref.py; "
                  "Res64 derived from its residue dump; dump_sha256 = SHA-256 of that dump file "
                  "(LucasNTT_results.dat, 19-byte records)",
        "cases": cases})


def make_ref_timings() -> None:
    """Per-iteration times of the reference build at each NTT length, from the
    oracle/run_ref.py summaries collected on a B200 (gpurun_out/ref_*/run_*.json).
    bench.py uses them to state the reference's plain one-at-a-time tests/hour."""
    base = ROOT / "gpurun_out"
    by_n = {}
    for js in sorted(base.glob("ref_*/run_*.json")):
        r = json.loads(js.read_text())
        if r.get("rc") != 0 or not r.get("per_iteration_ms"):
            continue
        by_n.setdefault(str(r["n"]), []).append({"q": r["exponent"], "prp": r["prp"], "pool": r["pool"],
                                                 "fft": r["fft_used"], "per_iteration_us": r["per_iteration_ms"] * 1e3})
    write("ref_timings.json", {
        "source": "reference LucasNTT build (oracle/build_ref.sh) run on a B200 by oracle/run_ref.py; "
                  "its own 'Per iteration (ms)' (lucas_prp.cu:319)",
        "by_n": by_n})


if __name__ == "__main__":
    sets = sys.argv[1:] or ["small"]
    for s in sets:
        if s == "small":
            make_small()
        elif s == "c1":
            make_c1()
        elif s == "c2":
            make_c2("--c2-long" in sets)
        elif s == "ref":
            make_ref()
        elif s == "reftimes":
            make_ref_timings()
