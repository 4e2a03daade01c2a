"""Extracts the reference's Turquin energy table (src/gpu/ggx_energy.cuh: E_ss(mu, r) of a white GGX conductor,
32 x 32, [j * 32 + i] for r = j/31 and sqrt(mu) = i/31) into tests/golden/ggx_energy_reference.txt, one value per
line, as the known answer the oracle's and the library's own quadratures are checked against. Run in a checkout that
has the reference: python tests/golden/make_ggx_energy_fixture.py [/path/to/reference] (default: $RT_REFERENCE_ROOT,
else a folder named `reference` beside this repository's checkout).
"""
import os
import re
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[2]
reference = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("RT_REFERENCE_ROOT", REPO.parent / "reference"))
text = (reference / "src" / "gpu" / "ggx_energy.cuh").read_text()
body = text[text.index("ggx_energy_table[") :]
body = body[body.index("{") + 1 : body.index("};")]
body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
values = [float(v.strip().rstrip("f")) for v in body.split(",") if v.strip()]
assert len(values) == 1024, len(values)
out = Path(__file__).resolve().parent / "ggx_energy_reference.txt"
out.write_text("".join(f"{v!r}\n" for v in values))
print(f"wrote {out} ({len(values)} values)")
