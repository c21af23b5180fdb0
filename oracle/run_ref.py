"""Run the reference's own build (oracle/_ref/LucasNTT) on a B200 and collect
its residue dump and timing.

Test infrastructure: pins residues against the reference build and measures its
"Per iteration (ms)" (lucas_prp.cu:319).  Usage (on a GPU box):

  python oracle/run_ref.py --exponent Q --iterations K [--fft N] [--prp]
                           [--loops 500] --out OUTDIR
  python oracle/run_ref.py --cases CASES.json [--loops 500] --out OUTDIR

CASES.json is a list of {"q", "iterations", "prp", "fft"} objects (written by
tests/golden/make_golden.py refcases); the cases run one after another and a
case whose summary already exists in OUTDIR is skipped, so an interrupted list
can be resumed.  Only the dumps' Res64 and SHA-256 are kept in this mode.
tests/golden/make_golden.py ref OUTDIR collects the summaries.

The program reads LucasNTT.ini from its working directory (main_process.cu:72)
and takes `exponent iterations fileprefix fft` on the command line
(main_process.cu:89-126); a forced non-optimal fft asks Y/N on stdin
(main_process.cu:136-141), answered "Y".  The dump (one 0x%016X word per line,
lucas_prp.cu:254-263) is renamed <q>_<n>_<prp>_<iterations>.dat.
"""
from __future__ import annotations

import argparse
import json
import re
import subprocess
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
BIN = HERE / "_ref" / "LucasNTT"


def summarize_dump(dat: Path, exponent: int, n: int):
    """Res64 (low 64 bits of sum d_j 2^ceil(q j / n)) of a residue dump."""
    import hashlib

    raw = dat.read_bytes()
    words = raw.split()
    r, pos = 0, 0
    for j, tok in enumerate(words):
        if pos >= 64:
            break
        r = (r + (int(tok, 16) << pos)) & 0xFFFFFFFFFFFFFFFF
        pos += -((-exponent * (j + 1)) // n) + ((-exponent * j) // n)  # width of word j
    return f"{r:016x}", len(words), hashlib.sha256(raw).hexdigest()


def run(exponent: int, iterations: int, out: Path, fft: str | None = None, prp: bool = False,
        loops: int = 500, timeout: int = 1800, keep_dump_bytes: int = 1 << 20) -> dict:
    out.mkdir(parents=True, exist_ok=True)
    (out / "LucasNTT.ini").write_text(
        "Verbosity = Normal\n"
        f"PerformanceLoops = {loops}\n"
        f"PRP = {1 if prp else 0}\n"
        "dumpResidue = 1\ndumpStats = 1\ndumpEnvironment = 1\n")
    prefix = f"run_{exponent}_{iterations}_{int(prp)}"
    for ext in (".dat", ".txt", ".env"):
        (out / (prefix + ext)).unlink(missing_ok=True)
    args = [str(BIN), str(exponent), str(iterations), prefix] + ([fft] if fft else [])
    t0 = time.time()
    r = subprocess.run(args, cwd=out, input="Y\n", capture_output=True, text=True, timeout=timeout)
    wall = time.time() - t0
    (out / (prefix + ".log")).write_text(r.stdout + r.stderr)
    stats = {}
    txt = out / (prefix + ".txt")
    if txt.exists():
        for line in txt.read_text().splitlines():
            if "=" in line:
                k, v = line.split("=", 1)
                stats[k.strip()] = v.strip()
    n = int(stats.get("n", "0"))
    dat = out / (prefix + ".dat")
    res64, words, digest = None, 0, None
    if dat.exists() and n:
        res64, words, digest = summarize_dump(dat, exponent, n)
        if dat.stat().st_size > keep_dump_bytes:
            dat.unlink()  # large dumps stay on the box; their Res64 and digest are kept
        else:
            dat.rename(out / f"{exponent}_{n}_{int(prp)}_{iterations}.dat")
    res = {"exponent": exponent, "iterations": iterations, "prp": prp, "fft": fft, "rc": r.returncode,
           "wall_s": wall, "n": n, "pool": stats.get("Pool"), "fft_used": stats.get("fft"),
           "per_iteration_ms": float(stats["Per iteration (ms)"]) if "Per iteration (ms)" in stats else None,
           "conclusion": stats.get("Conclusion"), "res64": res64, "words": words,
           "sha256_of_dump": digest,
           "kernels": [v for k, v in stats.items() if re.fullmatch(r"Kernel\d+", k)]}
    (out / (prefix + ".json")).write_text(json.dumps(res, indent=1))
    return res


def run_cases(cases_file: Path, out: Path, loops: int) -> None:
    cases = json.loads(cases_file.read_text())
    t0 = time.time()
    for i, c in enumerate(cases):
        q, prp = int(c["q"]), bool(c["prp"])
        it = int(c.get("iterations") or (q if prp else q - 2))
        if (out / f"run_{q}_{it}_{int(prp)}.json").exists():
            continue
        r = run(q, it, out, c.get("fft"), prp, loops, keep_dump_bytes=0)
        print(f"[{i + 1}/{len(cases)} {time.time() - t0:.0f}s] q={q} it={it} prp={int(prp)} n={r['n']} "
              f"rc={r['rc']} res64={r['res64']} wall={r['wall_s']:.1f}s", flush=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases")
    ap.add_argument("--exponent", type=int)
    ap.add_argument("--iterations", type=int, default=0)
    ap.add_argument("--fft")
    ap.add_argument("--prp", action="store_true")
    ap.add_argument("--loops", type=int, default=500)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    if a.cases:
        run_cases(Path(a.cases), Path(a.out), a.loops)
        raise SystemExit(0)
    it = a.iterations or (a.exponent if a.prp else a.exponent - 2)
    print(json.dumps(run(a.exponent, it, Path(a.out), a.fft, a.prp, a.loops)))
