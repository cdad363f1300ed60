"""Source check of the replayed time step's programmatic dependent launches (no GPU).

A kernel started by `launch_dep` (delta_b200/csrc/pdl.cuh) may begin while the kernel
before it on the stream is still running; it is correct only because its first statement,
`dep_sync()`, waits for that kernel's completion before anything is read or written. A
kernel that skipped it would race with its predecessor only under some timings, which a
GPU test may not catch. This test parses the CUDA sources: every kernel passed to
`launch_dep` (directly, or through a variable chosen among template instances) has
`dep_sync();` as the first statement of its body.
"""
import re
from pathlib import Path

CSRC = Path(__file__).resolve().parents[1] / "delta_b200" / "csrc"


def _sources():
    return {p.name: p.read_text() for p in sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh"))}


def _launched_kernels(sources):
    """Names of the kernels given to launch_dep, with the file of each launch."""
    out = set()
    for name, text in sources.items():
        if name == "pdl.cuh":
            continue
        for m in re.finditer(r"\blaunch_dep\(\s*[^,]+,\s*([A-Za-z_]\w*)", text):
            ident = m.group(1)
            if ident.startswith("k_"):
                out.add(ident)
                continue
            # a variable holding one of several kernels: every kernel named where it is set
            d = re.search(r"\bauto\s+" + ident + r"\s*=([^;]*);", text)
            assert d, f"{name}: launch_dep of {ident}, whose kernels are not found"
            kernels = set(re.findall(r"\b(k_\w+)\s*<", d.group(1))) | set(re.findall(r"\b(k_\w+)\b", d.group(1)))
            assert kernels, f"{name}: {ident} names no kernel"
            out |= kernels
    return out


def _first_statement(text, kernel):
    """The first statement of the body of __global__ kernel `kernel` in text, or None."""
    m = re.search(r"__global__[^;{]*?\b" + kernel + r"\s*\(", text)
    if not m:
        return None
    depth, j = 1, m.end()
    while depth:
        depth += {"(": 1, ")": -1}.get(text[j], 0)
        j += 1
    body = text.index("{", j)
    return text[body + 1:].lstrip().split(";", 1)[0] + ";"


def test_every_dependent_launch_waits_for_its_predecessor_first():
    sources = _sources()
    kernels = _launched_kernels(sources)
    assert {"k_cull_pairs", "k_cert_survivors", "k_bodies", "k_step_end", "k_skin_compact_block"} <= kernels
    for k in sorted(kernels):
        firsts = [s for s in (_first_statement(t, k) for t in sources.values()) if s is not None]
        assert firsts, f"kernel {k} not found"
        for f in firsts:
            assert f == "dep_sync();", f"{k}: first statement is {f!r}, not dep_sync();"
