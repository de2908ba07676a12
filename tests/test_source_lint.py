"""CPU: the library's sources issue no legacy-stream uploads or memsets.

A plain cudaMemcpy from host memory may return before its DMA lands, and
cudaMemset is asynchronous; both run on the legacy default stream, which
kernels on the handles' non-blocking streams are not ordered after.  Every
upload and memset therefore goes through a stream (the handle's), and this
test keeps it that way.  Device-to-host reads after a stream synchronize
are fine and are not flagged.
"""
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                    "wavefront_b200", "csrc")


def _calls(src: str, name: str):
    """(line, full argument text) of every call of `name` (multi-line aware)."""
    out = []
    for m in re.finditer(r"\b" + name + r"\s*\(", src):
        depth, i = 1, m.end()
        while depth and i < len(src):
            depth += {"(": 1, ")": -1}.get(src[i], 0)
            i += 1
        out.append((src.count("\n", 0, m.start()) + 1, src[m.end():i - 1]))
    return out


def _code(path: str) -> str:
    """The source with comments and string literals blanked out."""
    s = open(path).read()
    s = re.sub(r"//[^\n]*", "", s)
    s = re.sub(r"/\*.*?\*/", lambda m: "\n" * m.group(0).count("\n"), s, flags=re.S)
    return re.sub(r'"(\\.|[^"\\])*"', '""', s)


def test_no_legacy_stream_uploads_or_memsets():
    bad = []
    for f in sorted(os.listdir(CSRC)):
        if not f.endswith((".cu", ".cuh", ".cpp", ".h")):
            continue
        src = _code(os.path.join(CSRC, f))
        for line, args in _calls(src, "cudaMemcpy"):
            if "DeviceToHost" not in args:
                bad.append(f"{f}:{line}: cudaMemcpy({' '.join(args.split())[:60]})")
        for line, args in _calls(src, "cudaMemset"):
            bad.append(f"{f}:{line}: cudaMemset({' '.join(args.split())[:60]})")
    assert not bad, "legacy-stream uploads or memsets:\n" + "\n".join(bad)


def test_the_scanner_sees_calls():
    sample = "x(); cudaMemcpy(a, b,\n n, cudaMemcpyHostToDevice); cudaMemset(p, 0, 4);"
    assert [a.split(",")[-1].strip() for _, a in _calls(sample, "cudaMemcpy")] == [
        "cudaMemcpyHostToDevice"]
    assert len(_calls(sample, "cudaMemset")) == 1
    assert _calls("cudaMemsetAsync(p, 0, 4, s);", "cudaMemset") == []
