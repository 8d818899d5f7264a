"""Extract the CONF.INP sample that the reference's pconf documentation shows
(docs/pci/pconf.rst, the code block after "sample of the head of a
CONF.INP") into conf_inp_doc_head.txt, the block's indentation removed so
that the fixed columns of the file are as pconf reads them.

Run in a tree where the reference is present:
    python tests/golden/make_conf_inp_fixture.py /path/to/reference
"""
import pathlib
import sys
import textwrap


def extract(rst_text):
    lines = rst_text.splitlines()
    start = next(i for i, l in enumerate(lines) if "sample of the head of a" in l)
    k = next(i for i in range(start, len(lines)) if lines[i].strip().startswith(".. code-block::")) + 1
    while not lines[k].strip():
        k += 1
    block = []
    # the block runs while its lines are indented (or blank)
    while k < len(lines) and (lines[k].startswith(" ") or not lines[k].strip()):
        block.append(lines[k])
        k += 1
    while block and not block[-1].strip():
        block.pop()
    return textwrap.dedent("\n".join(block)) + "\n"


def main():
    ref = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "../reference")
    text = extract((ref / "docs" / "pci" / "pconf.rst").read_text())
    out = pathlib.Path(__file__).with_name("conf_inp_doc_head.txt")
    out.write_text(text)
    print(f"wrote {out} ({len(text.splitlines())} lines)")


if __name__ == "__main__":
    main()
