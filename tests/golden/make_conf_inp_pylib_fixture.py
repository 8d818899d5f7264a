"""Configuration lines of CONF.INP written by the reference's own Python
tools (py-lib/orbitals.py: convert_list_nr_to_rel_configs, which expands
non-relativistic configurations into relativistic ones, and
write_rel_configs, which create_conf_inp.py uses to write them), for a few
non-relativistic configurations, into conf_inp_pylib.txt; the expected
decoding, from py-lib's own convert_digital_to_char, and the group sizes
(relativistic configurations per non-relativistic one) into
conf_inp_pylib.json.

Run in a tree where the reference is present:
    python tests/golden/make_conf_inp_pylib_fixture.py /path/to/reference
"""
import io
import json
import pathlib
import sys

NR_CONFIGS = ["4f14", "4f13 5d1", "4f12 5d2", "4f13 6s1", "4f12 5d1 6p1", "4f13 10s1"]
NE = 14
HEADER = """  pylib test
  Z = 70.0
 Am = 173.0
  J =  0.0
 Jm =  0.0
 Nso=  0
 Nc = {nc}
 Kv =  4
 Nlv=  5
 Ne =  {ne}
"""


def main():
    ref = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "../reference")
    sys.path.insert(0, str(ref / "py-lib"))
    import orbitals as orb

    nrel, rel = orb.convert_list_nr_to_rel_configs(NR_CONFIGS)
    buf = io.StringIO()
    orb.write_rel_configs(rel, buf)
    text = HEADER.format(nc=nrel, ne=NE) + "\n" + buf.getvalue()
    expected = {"nr_configs": NR_CONFIGS, "group_sizes": [len(r) for r in rel], "configs": []}
    for nr_config in rel:
        for rc in nr_config:
            shells = []
            for code in orb.flatten_list(rc):
                if code[-1] == "0":              # write_rel_configs leaves these out
                    continue
                name, j = orb.convert_digital_to_char(code.strip())
                shells.append([name, j, int(code[-2:])])
            expected["configs"].append(shells)
    here = pathlib.Path(__file__).parent
    (here / "conf_inp_pylib.txt").write_text(text)
    (here / "conf_inp_pylib.json").write_text(json.dumps(expected, indent=1) + "\n")
    print(f"{nrel} relativistic configurations written")


if __name__ == "__main__":
    main()
