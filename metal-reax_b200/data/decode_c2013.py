#!/usr/bin/env python3
"""Extracts the carbon ReaxFF parameter set "Reactive MD-force field: 2013 C" (Srinivasan, van Duin, Ganesh, J. Phys.
Chem. A 119, 571 (2015)) from its Supporting Information PDF into a LAMMPS ffield file.

The parameters are not redistributed with this repository: the file is written into metal-reax_b200/data/_c2013/
(git-ignored) from a copy of the PDF the user provides, as the reference's examples/graphitization/make_ffield.sh does
with pdftotext. This script needs no external tool: the PDF's single page is one FlateDecode content stream of
monospaced text (a Type0 font with an Identity-H encoding and a ToUnicode map), so decoding it means inflating the
streams, mapping the glyph codes of every Tj string through the ToUnicode map, and starting a new line at every text
move with a vertical component.

    python decode_c2013.py <jp510274e_si_001.pdf> [output path]
"""
import re
import sys
import zlib
from pathlib import Path

HERE = Path(__file__).resolve().parent
DEFAULT_OUT = HERE / "_c2013" / "ffield.reax.C2013"


def _streams(data):
    """{object number: inflated stream bytes} of every FlateDecode stream."""
    out = {}
    for m in re.finditer(rb"(\d+) 0 obj\s*<<(.*?)>>\s*stream\r?\n", data, re.S):
        start = m.end()
        end = data.find(b"endstream", start)
        if b"FlateDecode" not in m.group(2):
            continue
        try:
            out[int(m.group(1))] = zlib.decompress(data[start:end])
        except zlib.error:
            continue
    return out


def _to_unicode(cmap):
    table = {}
    text = cmap.decode("latin-1")
    for block in re.findall(r"beginbfchar(.*?)endbfchar", text, re.S):
        for src, dst in re.findall(r"<([0-9a-fA-F]+)>\s*<([0-9a-fA-F]+)>", block):
            table[int(src, 16)] = chr(int(dst, 16))
    for block in re.findall(r"beginbfrange(.*?)endbfrange", text, re.S):
        for lo, hi, dst in re.findall(r"<([0-9a-fA-F]+)>\s*<([0-9a-fA-F]+)>\s*<([0-9a-fA-F]+)>", block):
            for k in range(int(lo, 16), int(hi, 16) + 1):
                table[k] = chr(int(dst, 16) + k - int(lo, 16))
    return table


def decode(pdf_bytes):
    streams = _streams(pdf_bytes)
    cmaps = [s for s in streams.values() if b"begincmap" in s]
    if not cmaps:
        raise ValueError("no ToUnicode map in the PDF")
    table = {}
    for c in cmaps:
        table.update(_to_unicode(c))
    lines = []
    for num in sorted(streams):
        content = streams[num]
        if b"BT" not in content or b"Tj" not in content:
            continue
        cur = []
        for tok in re.finditer(rb"<([0-9a-fA-F]*)>\s*Tj|(-?[\d.]+)\s+(-?[\d.]+)\s+Td|BT|ET", content):
            if tok.group(1) is not None:
                hexs = tok.group(1).decode()
                cur.append("".join(table.get(int(hexs[k:k + 4], 16), "?") for k in range(0, len(hexs), 4)))
            elif tok.group(2) is not None:
                if float(tok.group(3)) != 0.0:   # a move down: the next line
                    lines.append("".join(cur).rstrip())
                    cur = []
            elif tok.group(0) == b"ET" and cur:
                lines.append("".join(cur).rstrip())
                cur = []
        if cur:
            lines.append("".join(cur).rstrip())
    return "\n".join(lines) + "\n"


def main():
    if len(sys.argv) < 2:
        print(__doc__)
        sys.exit(1)
    out = Path(sys.argv[2]) if len(sys.argv) > 2 else DEFAULT_OUT
    text = decode(Path(sys.argv[1]).read_bytes())
    if "Reactive MD-force field: 2013 C" not in text:
        print("unexpected content: this is not the 2013 C force field", file=sys.stderr)
        sys.exit(2)
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_text(text)
    print("wrote %s (%d lines)" % (out, text.count("\n")))


if __name__ == "__main__":
    main()
