"""Writes sobol_directions.json: the sampler's direction numbers as the reference holds them.

The reference's kernel sampler (renderer/shaders/sample.wgsl:5-64) unrolls the first 16 bit-reversed direction
numbers of Sobol dimensions 1-3 as hex literals, and its CPU mirror's test (renderer/src/sample.rs:90-99,
`the_directions_are_the_shaders`) holds the 32-entry tables to those literals and their last entries to
0xffffffff, 0xaaaa00a3, 0xc900a00a. This script reads the literals out of the WGSL text so the oracle's own
recurrence is checked against the reference's numbers. Run it where the reference is mounted, with the path of
renderer/shaders/sample.wgsl as its one argument; its output is committed.

  python tests/golden/make_sobol_fixture.py <reference>/renderer/shaders/sample.wgsl
"""
import json
import re
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit(__doc__)
src = Path(sys.argv[1]).read_text()
dims = []
for name in ("sobol_d1", "sobol_d2", "sobol_d3"):
    body = src.split(f"fn {name}(x: u32) -> u32 {{", 1)[1].split("return r;", 1)[0]
    vals = [int(v, 16) for v in re.findall(r"select\(0u, 0x([0-9a-f]{8})u", body)]
    assert len(vals) == 16, name
    dims.append(vals)
out = {"first16": dims, "last": [0xFFFFFFFF, 0xAAAA00A3, 0xC900A00A],
       "source": "renderer/shaders/sample.wgsl:5-64; renderer/src/sample.rs:98"}
Path(__file__).with_name("sobol_directions.json").write_text(json.dumps(out, indent=1) + "\n")
print("wrote", len(dims), "dimensions")
