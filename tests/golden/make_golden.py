"""Copy the reference's own golden vectors for the propagation path into
tests/golden/ (run once, where the reference is mounted; its directory is the first
argument or EDUS_REFERENCE_DIR).

Sources (gcistaro/EDUS_2.0):
  ci-test/outputs/hBN/{Population,Velocity,Laser,Time}.txt
      output of the hBN IPA integration test (ci-test/inputs/hBN.json.in,
      tb_models/hBN_gap7.25eV_a2.5A_tb.dat), compared by ci-test/compare.py
      at 1e-10 absolute (column 0 skipped);
  ci-test/Reference/Struve.txt
      Struve H_v(x) table, x = -5..5, used for the screened potential.
The files are copied byte for byte; tests read them with numpy.loadtxt.
"""
import os
import shutil
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("EDUS_REFERENCE_DIR", "")
if not os.path.isdir(os.path.join(REF, "ci-test")):
    raise SystemExit("usage: make_golden.py <reference dir> (or set EDUS_REFERENCE_DIR)")
HERE = os.path.dirname(os.path.abspath(__file__))

os.makedirs(os.path.join(HERE, "hBN"), exist_ok=True)
for name in ("Population", "Velocity", "Laser", "Time"):
    shutil.copyfile(os.path.join(REF, "ci-test", "outputs", "hBN", name + ".txt"),
                    os.path.join(HERE, "hBN", name + ".txt"))
shutil.copyfile(os.path.join(REF, "ci-test", "Reference", "Struve.txt"), os.path.join(HERE, "Struve.txt"))
print("golden vectors written to", HERE)
