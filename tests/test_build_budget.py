"""Register budget of the hot kernels, read from the build's `-Xptxas -v` reports.

The force kernels keep several CTAs resident per SM through `__launch_bounds__` (the Hermite
j-paired forms: three 128-thread CTAs, at most 168 registers a thread).  ptxas meets such a
bound by spilling, so a source change that needs more registers shows up here as spill stores
before it shows up on a GPU as a slower pair loop.  No GPU is needed: the reports are written
by `make` next to the libraries (lib/*.ptxas.txt).
"""
import os
import re

import pytest

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "phantom-grape_b200", "lib")


def ptxas_report(name):
    """{mangled entry name: (registers, spill store bytes)} of one library's ptxas report."""
    path = os.path.join(LIB, name + ".ptxas.txt")
    if not os.path.exists(path):
        pytest.skip(f"{name}.ptxas.txt not built")
    out, cur, regs = {}, None, None
    for line in open(path):
        m = re.search(r"Compiling entry function '(\S+)'", line)
        if m:
            cur, regs = m.group(1), None
            continue
        m = re.search(r"Used (\d+) registers", line)
        if m and cur:
            regs = int(m.group(1))
            out[cur] = (regs, out.get(cur, (None, 0))[1])
        m = re.search(r"(\d+) bytes spill stores", line)
        if m and cur:
            out[cur] = (out.get(cur, (regs, 0))[0], int(m.group(1)))
    assert out, f"no entry functions in {path}"
    return out


# g6_kernel<NT, IPT, JL, FF, NN, NBL, JP> with JP = 1 (j-pair order) or 2 (stage-ordered):
# the configurations the autotuner picks from 2048 active particles up
JPAIRED = re.compile(r"_ZN3pgb9g6_kernelILi(\d+)ELi(\d+)ELi1ELb1ELb([01])ELb0ELi([12])EEEv")


@pytest.mark.parametrize("lib", ["libpg6", "libpg6_newton"])
def test_hermite_j_paired_kernels_do_not_spill(lib):
    rep = ptxas_report(lib)
    hits = {k: v for k, v in rep.items() if JPAIRED.match(k)}
    assert len(hits) >= 4, f"j-paired Hermite kernels not found in {lib}: {sorted(rep)[:5]}"
    for k, (regs, spill) in hits.items():
        nt, ipt = map(int, JPAIRED.match(k).group(1, 2))
        assert spill == 0, f"{lib} {k}: {spill} bytes of spill stores"
        if nt == 128 and ipt == 2:
            # three CTAs of 128 threads on an SM's 65536 registers (allocated in units of 8)
            assert regs <= 168, f"{lib} {k}: {regs} registers, above the 3-CTA budget"


@pytest.mark.parametrize("lib", ["libpg5", "libpg5sym", "libpg5table", "libpgbpeak"])
def test_pg5_and_peak_kernels_do_not_spill(lib):
    rep = ptxas_report(lib)
    spilled = {k: s for k, (_, s) in rep.items() if s}
    assert not spilled, f"{lib}: spill stores in {spilled}"


@pytest.mark.parametrize("lib", ["libpg6", "libpg6_newton"])
def test_drop_in_kernels_stay_within_their_two_cta_budget(lib):
    """The drop-in API's small-call kernel runs two 512-thread CTAs an SM (its clusters must all
    be resident at once), so ptxas caps it at 64 registers; the few words it spills stay in L1.
    The bound here is today's spill (12 bytes a thread, 60 for the 32 x 16 shape) with room for
    one more double, not a license to grow it."""
    rep = ptxas_report(lib)
    small = {k: v for k, v in rep.items() if k.startswith("_ZN3pgb15g6_small_kernel")}
    assert len(small) >= 16, f"small-call kernels not found in {lib}"
    for k, (regs, spill) in small.items():
        assert regs <= 64, f"{lib} {k}: {regs} registers, above two 512-thread CTAs an SM"
        assert spill <= 68, f"{lib} {k}: {spill} bytes of spill stores"
