"""GPU: the lucasntt program as a drop-in for the reference's command line.

Same LucasNTT.ini keys and argv, same console verdicts, and result files the
reference can read: the residue dump of a run is byte-for-byte the file the
reference build wrote for the same test (SHA-256 in tests/golden/ref_residues.json).
Interruption (SIGINT), a crash after a safety dump (SIGKILL of the host
process between chunks of squarings) and a corrupt dump are recovered as the
reference does (main_process.cu:98-118, lucas_prp.cu:137-150, :326-346).
"""
import hashlib
import json
import signal
import subprocess
import time
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
BIN = ROOT / "cuda_b200" / "lucasntt"
REF = json.loads((ROOT / "tests" / "golden" / "ref_residues.json").read_text())["cases"]


@pytest.fixture(scope="module", autouse=True)
def built():
    if not BIN.exists():
        subprocess.run(["make", "-C", str(ROOT / "cuda_b200"), "lucasntt"], check=True)


def run_cli(cwd, args, ini=None, stdin="", timeout=900):
    if ini is not None:
        (cwd / "LucasNTT.ini").write_text(ini)
    return subprocess.run([str(BIN), *map(str, args)], cwd=cwd, capture_output=True, text=True,
                          input=stdin, timeout=timeout)


def stats(path: Path) -> dict:
    out = {}
    for line in path.read_text().splitlines():
        if " = " in line:
            k, v = line.split(" = ", 1)
            out[k.strip()] = v.strip()
    return out


def sha256(path: Path) -> str:
    return hashlib.sha256(path.read_bytes()).hexdigest()


def direct_res64(lnt, q, iterations, prp=False):
    with lnt.LucasTest(q, prp=prp) as t:
        t.iterate(iterations)
        return f"{t.res64():016X}"


def test_full_ll_known_prime(tmp_path):
    r = run_cli(tmp_path, [9689], ini="PerformanceLoops = 50\n")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "M(9689) is prime!" in r.stdout
    s = stats(tmp_path / "LucasNTT_results.txt")
    assert s["Conclusion"] == "Prime" and s["Interrupted"] == "0" and s["currentIteration"] == "9688"
    assert s["Res64"] == "0000000000000000" and s["fft"] == "512" and s["PRP"] == "0"
    assert not (tmp_path / "LucasNTT_results.dat").exists()  # full test, dumpResidue = 0


def test_full_prp_probable_prime_and_environment(tmp_path):
    r = run_cli(tmp_path, [], ini="Exponent = 9941\nPRP = 1\nPerformanceLoops = 50\ndumpEnvironment = 1\n")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "M(9941) is probably prime!" in r.stdout
    s = stats(tmp_path / "LucasNTT_results.txt")
    assert s["Conclusion"] == "Probably Prime" and s["Res64"] == "0000000000000009"
    env = (tmp_path / "LucasNTT_results.env").read_text()
    assert "CUDA Version = " in env and "Device 0 = " in env and "Multiprocessors = " in env


def test_gerbicz_check_from_the_ini(tmp_path):
    """GerbiczBlock (an extension key): a checked PRP of M_132049, checks in the stats file."""
    r = run_cli(tmp_path, [132049, 0, "g"], ini="PRP = 1\nPerformanceLoops = 50\nGerbiczBlock = 64\n")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "M(132049) is probably prime!" in r.stdout
    s = stats(tmp_path / "g.txt")
    # every block of 64^2 squarings verified; errors (each recovered) depend on the hardware
    assert s["Gerbicz checks"] == str(132049 // 4096) and int(s["Gerbicz errors"]) >= 0


def test_composite_verdict(tmp_path):
    r = run_cli(tmp_path, [9973, 0, "c"], ini="PerformanceLoops = 50\n")
    assert r.returncode == 0 and "M(9973) is composite!" in r.stdout
    assert stats(tmp_path / "c.txt")["Conclusion"] == "Composite"


@pytest.mark.parametrize("case", [c for c in REF if c["n"] <= 4096],
                         ids=lambda c: f"{c['q']}@{c['n']}{'_prp' if c['prp'] else ''}")
def test_dump_file_equals_reference_c1(tmp_path, case):
    """Full LL and PRP tests with dumpResidue = 1 (the C1 exponents, the
    serving stream's small exponents, PRP fulls): the .dat file is the
    reference's, byte for byte."""
    args = [case["q"], case["iterations"], "run"]
    if case["q"] in (44497, 44501, 44507, 44519, 44531, 44533, 44537, 44543, 44549) and case["n"] == 4096:
        args.append(case["n"])  # the forced length 4096 needs the fft argument
    prp = "PRP = 1\n" if case["prp"] else ""
    r = run_cli(tmp_path, args, ini=prp + "dumpResidue = 1\nPerformanceLoops = 100\n", stdin="Y\n")
    assert r.returncode == 0, r.stdout + r.stderr
    s = stats(tmp_path / "run.txt")
    assert s["n"] == str(case["n"])
    assert s["Res64"].lower() == case["res64"]
    assert sha256(tmp_path / "run.dat") == case["dump_sha256"]


@pytest.mark.parametrize("case", [c for c in REF if c["n"] == 1 << 23],
                         ids=lambda c: f"{c['iterations']}{'_prp' if c['prp'] else ''}")
def test_dump_file_equals_reference_c2(tmp_path, case):
    """q = 139000003 at 2^23, LL and PRP: a partial run always dumps
    (lucas_prp.cu:189); same bytes."""
    prp = "PRP = 1\n" if case["prp"] else ""
    r = run_cli(tmp_path, [case["q"], case["iterations"], "c2"], ini=prp + "PerformanceLoops = 100\n")
    assert r.returncode == 0, r.stdout + r.stderr
    assert f"{case['iterations']} loops performed with M({case['q']})" in r.stdout
    s = stats(tmp_path / "c2.txt")
    assert s["Conclusion"] == "Partial" and s["Interrupted"] == "0"
    assert s["currentIteration"] == str(case["iterations"] + 1)
    assert sha256(tmp_path / "c2.dat") == case["dump_sha256"]


def start(cwd, args, ini):
    (cwd / "LucasNTT.ini").write_text(ini)
    return subprocess.Popen([str(BIN), *map(str, args)], cwd=cwd, stdout=subprocess.PIPE,
                            stderr=subprocess.STDOUT, text=True)


def wait_for_line(p, text, timeout=300):
    t0 = time.time()
    lines = []
    while time.time() - t0 < timeout:
        line = p.stdout.readline()
        if not line:
            break
        lines.append(line)
        if text in line:
            return lines
    raise AssertionError(f"'{text}' not seen: {''.join(lines)[-2000:]}")


Q_LONG, IT_LONG = 1000003, 400000  # several seconds of squarings at 64K words


def test_sigint_then_resume(tmp_path, lnt):
    p = start(tmp_path, [Q_LONG, IT_LONG, "run"], "PerformanceLoops = 50\n")
    wait_for_line(p, "From iteration")
    time.sleep(1.0)
    p.send_signal(signal.SIGINT)
    out, _ = p.communicate(timeout=300)
    assert p.returncode == 0, out
    s = stats(tmp_path / "run.txt")
    assert s["Interrupted"] == "1" and s["Conclusion"] == "Partial"
    stopped = int(s["currentIteration"])
    assert 1 < stopped <= IT_LONG
    assert (tmp_path / "run.dat").exists()
    r = run_cli(tmp_path, [Q_LONG, IT_LONG, "run"])
    assert r.returncode == 0, r.stdout
    assert "Last execution was interrupted" in r.stdout and "Previous residue successfully loaded!" in r.stdout
    assert f"From iteration {stopped} to {IT_LONG}" in r.stdout
    s = stats(tmp_path / "run.txt")
    assert s["Interrupted"] == "0" and s["currentIteration"] == str(IT_LONG + 1)
    assert s["Res64"] == direct_res64(lnt, Q_LONG, IT_LONG)


def test_crash_after_safety_dump_resumes(tmp_path, lnt):
    """The process dies (SIGKILL between chunks) after a safety dump; the next
    run resumes from that dump."""
    p = start(tmp_path, [Q_LONG, IT_LONG, "run"], "PerformanceLoops = 50\nSafetyDumpSeconds = 1\n")
    wait_for_line(p, "Now dumping intermediate residue")
    time.sleep(0.3)
    p.kill()
    p.communicate(timeout=60)
    s = stats(tmp_path / "run.txt")
    assert s["Interrupted"] == "1"
    dumped_at = int(s["currentIteration"])
    r = run_cli(tmp_path, [Q_LONG, IT_LONG, "run"])
    assert r.returncode == 0, r.stdout
    assert "Previous residue successfully loaded!" in r.stdout
    assert f"From iteration {dumped_at} to {IT_LONG}" in r.stdout
    assert stats(tmp_path / "run.txt")["Res64"] == direct_res64(lnt, Q_LONG, IT_LONG)


def test_corrupt_dump_restarts_from_one(tmp_path):
    (tmp_path / "LucasNTT_results.txt").write_text(
        "Exponent = 9689\nPRP = 0\nIterations = 9687\nInterrupted = 1\ncurrentIteration = 5000\n")
    (tmp_path / "LucasNTT_results.dat").write_text("0x0000000000000004\n0x00000000000")
    r = run_cli(tmp_path, [], ini="PerformanceLoops = 50\n")
    assert r.returncode == 0, r.stdout
    assert "Failed to restore previous residue, restarting from iteration 1!" in r.stdout
    assert "M(9689) is prime!" in r.stdout


def test_provided_length_prompt(tmp_path):
    r = run_cli(tmp_path, [44497, 100, "x", 1024], ini="PerformanceLoops = 50\n", stdin="N\n")
    assert r.returncode == 1 and "Process cancelled by user. Invalid FFT length." in r.stdout
    r = run_cli(tmp_path, [44497, 100, "x", 4096], stdin="Y\n")
    assert r.returncode == 0 and stats(tmp_path / "x.txt")["n"] == "4096"


def test_pool_preference(tmp_path, lnt):
    name = lnt.plan_describe((2, 7, 8), 1000003)  # a plan the policy would not pick
    r = run_cli(tmp_path, [1000003, 200, "p"], ini=f"PerformanceLoops = 50\nPool = {name}\n")
    assert r.returncode == 0, r.stdout
    assert stats(tmp_path / "p.txt")["Pool"] == name


def test_jacobi_check_from_the_ini(tmp_path):
    """JacobiCheck (an extension key): a checked LL test of M_132049, checks in the stats file."""
    r = run_cli(tmp_path, [132049, 0, "j"], ini="PerformanceLoops = 50\nJacobiCheck = 20000\n")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "M(132049) is prime!" in r.stdout
    s = stats(tmp_path / "j.txt")
    assert s["Jacobi checks"] == str((132049 - 2) // 20000) and s["Jacobi errors"] == "0"


def test_five_length_from_the_ini(tmp_path):
    """fft = 40960 (5 * 2^13): no reference kernel has it; the program asks as the
    reference does for a non-optimal length (this exponent's smallest is 16384),
    then runs the full LL test of the Mersenne prime M_216091 on it."""
    r = run_cli(tmp_path, [], ini="Exponent = 216091\nfft = 40960\nPerformanceLoops = 20\n", stdin="y\n")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "not optimal" in r.stdout and "M(216091) is prime!" in r.stdout
    s = stats(tmp_path / "LucasNTT_results.txt")
    assert s["Res64"] == "0000000000000000" and s["fft"] == "64:640"
