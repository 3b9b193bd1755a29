"""Extracts the reference's golden XDMF3 document from its writer test
(test/test_writers.jl of the FastIce.jl checkout given as the first argument) into
xdmf3_writers_ref.xml next to this script.  That test writes the metadata of two
Center fields "Fa", "Fb" on UniformGrid(origin=(-0.4, -0.5, 0.0), extent=(1.0,
1.1, 1.2), dims=(4, 5, 6)) for the HDF5 file "test.h5" at time 0.0.

    python tests/golden/make_golden_writers.py /path/to/FastIce.jl
"""
import os
import re
import sys

src = os.path.join(sys.argv[1], "test", "test_writers.jl")
text = open(src, encoding="utf-8").read()
m = re.search(r'XML_ref = """\n(.*?)"""', text, re.S)
if not m:
    raise SystemExit("XML_ref not found in " + src)
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "xdmf3_writers_ref.xml")
with open(out, "w", encoding="utf-8") as f:
    f.write(m.group(1))
print("wrote", out, len(m.group(1)), "bytes")
