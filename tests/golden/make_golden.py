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
  refcases  write ref_cases.json, the list of reference-build runs that pin
         PRP mode and the batch/serving exponents (run on a B200 by
         oracle/run_ref.py --cases tests/golden/ref_cases.json --out DIR)
  ref DIR...  merge the reference build's run summaries found in the given
         directories (run_*.json written by oracle/run_ref.py) into
         ref_residues.json (cases already there are kept)
  reftimes DIR...  the reference build's per-iteration times from the same
         summaries into ref_timings.json

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

from bench import c3_exponents, c4_exponents, c5_pool  # noqa: E402  (the workloads' seeded exponents)
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


C3_CHECK_ITERATIONS = 20000
C4_ITERATIONS = 20000
C5_FULL_LIMIT = 610000


def ref_cases() -> list[dict]:
    """Reference-build runs pinning PRP mode and the batch and serving exponents.

    C4: all 64 PRP tests at 20,000 squarings.  C3: a full LL test of the first
    sampled exponent of each length, and every one of the 256 exponents after
    20,000 squarings.  PRP: full tests of a composite and of Mersenne primes on
    both plan kinds, and q = 139000003 after 1,000 squarings.  C5: full tests of
    the pool's requests up to q = 610,000.  Large: 1,000 squarings at 2^24 (LL and
    PRP), 2^25 and 2^26."""
    from oracle import oracle as O

    cases = [{"q": q, "iterations": C4_ITERATIONS, "prp": True, "set": "c4"} for q in c4_exponents()]
    first = {}
    for q in c3_exponents():
        first.setdefault(1 << O.secured_log2(q), q)
    cases += [{"q": q, "iterations": q - 2, "prp": False, "set": "c3_full"} for _, q in sorted(first.items())]
    cases += [{"q": 100003, "iterations": 100003, "prp": True, "set": "prp"},
              {"q": 160001, "iterations": 160001, "prp": True, "set": "prp"},
              {"q": 132049, "iterations": 132049, "prp": True, "set": "prp"},
              {"q": 44497, "iterations": 44497, "prp": True, "set": "prp"},
              {"q": 44497, "iterations": 44497, "prp": True, "fft": "4096", "set": "prp"},
              {"q": 44501, "iterations": 44501, "prp": True, "set": "prp"},
              {"q": C2_EXPONENT, "iterations": 1000, "prp": True, "set": "prp"}]
    seen = set()
    for q, prp in sorted(c5_pool()):
        if q <= C5_FULL_LIMIT and (q, prp) not in seen:
            seen.add((q, prp))
            cases.append({"q": q, "iterations": q if prp else q - 2, "prp": prp, "set": "c5_full"})
    cases += [{"q": q, "iterations": C3_CHECK_ITERATIONS, "prp": False, "set": "c3_check"} for q in c3_exponents()]
    # the largest lengths (2^24, 2^25, 2^26: q = 300000007, 600000001, 1100000009), 1,000 squarings
    cases += [{"q": q, "iterations": 1000, "prp": prp, "set": "large"}
              for q, prp in ((300000007, False), (300000007, True), (600000001, False), (1100000009, False))]
    return cases


def make_ref_cases() -> None:
    write("ref_cases.json", ref_cases())


def _summaries(dirs: list[str]):
    for d in dirs:
        for js in sorted(Path(d).glob("run_*.json")):
            r = json.loads(js.read_text())
            if r.get("rc") == 0 and r.get("res64"):
                yield r


def make_ref(dirs: list[str]) -> None:
    """Merge the reference runs summarised by oracle/run_ref.py (run_*.json:
    Res64 of the reference's residue dump) into ref_residues.json.  A case whose
    double-precision widths start some word below its weight's bit carries
    "shifted_words" (their count): there the reference's sequence is not that of
    M_q, and true_residues.json holds the true Res64."""
    from cuda_b200 import shifted_words

    path = HERE / "ref_residues.json"
    old = json.loads(path.read_text())["cases"] if path.exists() else []
    key = lambda c: (c["q"], c["n"], c["prp"], c["iterations"])  # noqa: E731
    merged = {key(c): c for c in old}
    sets = {(c["q"], c["iterations"], c["prp"]): c["set"] for c in ref_cases()}
    for r in _summaries(dirs):
        c = {"q": r["exponent"], "n": r["n"], "prp": r["prp"], "iterations": r["iterations"],
             "res64": r["res64"], "fft": r["fft_used"], "pool": r["pool"],
             "per_iteration_ms": r["per_iteration_ms"], "conclusion": r["conclusion"],
             "dump_sha256": r.get("sha256_of_dump")}
        if (c["q"], c["iterations"], c["prp"]) in sets:
            c["set"] = sets[(c["q"], c["iterations"], c["prp"])]
        merged[key(c)] = c
    for c in merged.values():
        k = shifted_words(c["q"], c["n"])[0]
        if k:
            c["shifted_words"] = k
    write("ref_residues.json", {
        "source": "reference LucasNTT build (oracle/build_ref.sh) run on a B200 by oracle/run_ref.py; "
                  "Res64 derived from its residue dump; dump_sha256 = SHA-256 of that dump file "
                  "(19-byte records)",
        "cases": list(merged.values())})


def make_ref_timings(dirs: list[str]) -> None:
    """Per-iteration times of the reference build at each NTT length, from the
    oracle/run_ref.py summaries (run_*.json) in the given directories, merged
    into ref_timings.json.  bench.py uses them to state the reference's plain
    one-at-a-time tests/hour."""
    path = HERE / "ref_timings.json"
    by_n = json.loads(path.read_text())["by_n"] if path.exists() else {}
    for r in _summaries(dirs):
        if not r.get("per_iteration_ms"):
            continue
        rows = by_n.setdefault(str(r["n"]), [])
        row = {"q": r["exponent"], "prp": r["prp"], "pool": r["pool"], "fft": r["fft_used"],
               "per_iteration_us": r["per_iteration_ms"] * 1e3}
        if row not in rows:
            rows.append(row)
    write("ref_timings.json", {
        "source": "reference LucasNTT build (oracle/build_ref.sh) run on a B200 by oracle/run_ref.py; "
                  "its own 'Per iteration (ms)' (lucas_prp.cu:319)",
        "by_n": by_n})


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] in ("ref", "reftimes"):
        (make_ref if sys.argv[1] == "ref" else make_ref_timings)(sys.argv[2:])
        raise SystemExit(0)
    sets = sys.argv[1:] or ["small"]
    for s in sets:
        if s == "small":
            make_small()
        elif s == "c1":
            make_c1()
        elif s == "c2":
            make_c2("--c2-long" in sets)
        elif s == "refcases":
            make_ref_cases()
