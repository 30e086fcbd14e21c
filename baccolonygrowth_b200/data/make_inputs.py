"""Regenerate small_input.txt / large_input.txt from the reference's shipped
input files (run_sim/inputFile_20mM_{Small,Large}Simulation.txt): the
"key value" pairs only, in the reference's own key/value format, so that the
parameter sets travel with the package.  Run where the reference tree is
mounted:  python baccolonygrowth_b200/data/make_inputs.py <reference_dir>
(reference_dir = the AgentBasedModel-BacColonyGrowth directory; or set
BCG_REF_DIR to it).
"""
import os
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("BCG_REF_DIR", "")
if not REF:
    sys.exit("usage: make_inputs.py <AgentBasedModel-BacColonyGrowth directory> (or set BCG_REF_DIR)")
HERE = os.path.dirname(os.path.abspath(__file__))

for src, dst in (("inputFile_20mM_SmallSimulation.txt", "small_input.txt"),
                 ("inputFile_20mM_LargeSimulation.txt", "large_input.txt")):
    out = []
    with open(os.path.join(REF, "run_sim", src)) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] not in ("Restart_dir",):
                out.append("%s %s" % (parts[0], parts[1]))
    with open(os.path.join(HERE, dst), "w") as f:
        f.write("\n".join(out) + "\n")
    print("wrote", dst, len(out), "keys")
