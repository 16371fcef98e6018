"""Writes mqp_twiddles.inc: cos/sin(2*pi*m/256) for m in [0, 256), rounded
once from double to float.  Regenerate with ``python gen_twiddles.py``."""
import math, os
N = 256
rows = []
for m in range(N):
    a = 2.0 * math.pi * m / N
    c, s = math.cos(a), math.sin(a)
    if abs(c) < 1e-15: c = 0.0
    if abs(s) < 1e-15: s = 0.0
    rows.append("  {%.9ef, %.9ef}" % (c, s))
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mqp_twiddles.inc")
with open(out, "w") as f:
    f.write("// generated by gen_twiddles.py: {cos, sin}(2*pi*m/%d), m = 0..%d\n" % (N, N - 1))
    f.write(",\n".join(rows) + "\n")
