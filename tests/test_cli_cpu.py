"""The ltli6463-compatible command line on the host: its argument checks, the missing-file
and input-limit messages (all printed before any device call), and, on a host without a
CUDA device, the stdout layout that code/dc.py parses (ltli6463.cu:1580-1677)."""
import os
import subprocess

import pytest

from ltlb200 import api
from helpers import fixture_path

CLI = api.CLI_PATH
UNIT = ["1"] * 8


def run(*args):
    p = subprocess.run([CLI, *args], capture_output=True, text=True, timeout=60)
    assert p.returncode == 0  # the reference always exits 0 (ltli6463.cu:1589, :1608, :1612)
    return p.stdout


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


pytestmark = pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")


def test_usage_when_arguments_are_missing():
    out = run("x", *UNIT, "500", "3")
    lines = out.split("\n")
    assert lines[0] == "Arguments should be in the form of"
    assert lines[2].endswith(" <input_file_address> <c1> <c2> <c3> <c4> <c5> <c6> <c7> <c8> <maxCost> "
                             "<RlxUnqChkTyp> <NegType>")
    assert lines[5] == "For example"
    assert lines[7].endswith(" ./input.txt 1 1 1 1 1 1 1 1 500 3 2")


def test_argument_checks_in_reference_order():
    out = run("x", "0", "1", "1", "1", "1", "1", "1", "40000", "500", "4", "3")
    assert out == ('Argument number 2, "0", should be a positive short integer.\n'
                   'Argument number 9, "40000", should be a positive short integer.\n'
                   'Argument number 11, RlxUnqChkTyp = "4", should be 1, 2, or 3.\n'
                   'Argument number 12, NegType = "3", should be 1, or 2.\n')


def test_max_cost_is_a_positive_short():
    out = run("x", *UNIT, "0", "3", "2")
    assert out == 'Argument number 10, "0", should be a positive short integer.\n'


def test_unknown_trailing_flag_is_an_argument_error():
    out = run(fixture_path("ham1_len3.trace"), *UNIT, "500", "3", "2", "--bogus")
    assert out == 'Unknown option "--bogus".\n'


def test_missing_input_file():
    assert run("/nonexistent/input.trace", *UNIT, "500", "3", "2") == "Failed to open the input file.\n"


@pytest.mark.parametrize("flag,limit", [([], 8192), (["--limit-traces"], 64)])
def test_input_limits_are_reported_before_the_device(flag, limit):
    """A trace of 64 steps is refused with the reference's message and nothing else printed
    (the reference returns from main on "see_the_error", ltli6463.cu:1629)."""
    out = run(fixture_path("len64.trace"), *UNIT, "500", "3", "2", *flag)
    assert out == ("In this version, The input can have:\n"
                   f"1) At most {limit} traces. It is currently 6.\n"
                   "2) Max(len(trace)) = 63. It is currently 64.\n")


def expected_listing(text):
    """The trace listing of ltli6463.cu:1642-1666 from the file text: one line per trace, a
    tab, then "{letters}\\t" per time step, letters in the file's value order."""
    lines = text.split("\n")
    body = text[:-1] if text.endswith("\n") else text
    alpha = "".join(c for c in body.split("\n")[-1] if "a" <= c <= "z")
    sides, cur = [], []
    for ln in lines:
        if ln == "---":
            sides.append(cur)
            cur = []
            if len(sides) == 2:
                break
            continue
        cur.append(ln)
    out = []
    for title, side in zip(("Positive", "Negative"), sides):
        out.append(f"\n{title}: \n")
        for ln in side:
            steps = []
            for tok in ln.split(";"):
                vals = [c for c in tok if c != ","]
                steps.append("{" + ", ".join(alpha[j] for j, c in enumerate(vals) if c == "1" and j < len(alpha)) + "}")
            out.append("\t" + "".join(s + "\t" for s in steps) + "\n")
    return "".join(out)


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
@pytest.mark.parametrize("name", ["ham1_len3.trace", "f10x10_p3_s0.trace", "cfg1_s0.trace"])
def test_stdout_layout_without_a_device(name):
    """Traces, cost function and trace count as the reference prints them, the measurement
    lines, and the result line second to last (what dc.py reads, code/dc.py:194, :278); with
    no device the result is the status text, never a CPU-computed formula."""
    path = fixture_path(name)
    out = run(path, "1", "2", "1", "1", "1", "1", "1", "3", "500", "3", "2")
    text = open(path).read()
    listing = expected_listing(text)
    assert out.startswith(listing)
    rest = out[len(listing):].split("\n")
    npos = len(text.split("\n---\n")[0].split("\n"))
    nneg = len(text.split("\n---\n")[1].split("\n"))
    assert rest[1] == "Cost Function: p:1, ~:2, &:1, |:1, X:1, F:1, G:1, U:3"
    assert rest[2] == f"Number of Traces: {npos + nneg}"
    assert rest[3].startswith("Number of All LTLs: ")
    assert rest[4].startswith("Cost of Final LTL: ")
    assert rest[5].startswith("Running Time: ") and rest[5].endswith(" s")
    assert out.split("\n")[-2] == 'LTL: "no_cuda_device"'


def test_per_block_letters_line_matches_reference_runs():
    """With --per-block the first line is the letters' progress line, as the reference binary
    printed it in every recorded run (ltli6463.cu:1095-1098; printed before any device work)."""
    from helpers import reference_runs
    runs = reference_runs()
    if runs is None:
        pytest.skip("reference outputs not recorded")
    seen = 0
    for r in runs["runs"]:
        if r["final"]["limits_error"]:
            continue
        cost, op, all_before, stored, to_check = r["progress"][0]
        assert op == "A"
        p = subprocess.run([CLI, fixture_path(r["file"]), *[str(c) for c in r["costs"]], str(r["max_cost"]),
                            str(r["rlx"]), str(r["neg"]), "--per-block"], capture_output=True, text=True, timeout=300)
        first = p.stdout.split("\n")[0]
        assert first == (f"Cost {cost:<2d} | (A) | AllLTLs: {all_before:<11d} | StoredLTLs: {stored:<10d} | "
                         f"ToBeChecked: {to_check:<10d} "), (r["id"], first)
        seen += 1
    assert seen >= 70
