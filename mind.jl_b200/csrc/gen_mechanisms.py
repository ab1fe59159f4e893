"""Write generated_mechanisms.cuh: CUDA C emitted from MOD files by mind_b200.nmodl.

    python mind.jl_b200/csrc/gen_mechanisms.py [MOD_DIR] [extra.mod ...]

MOD_DIR defaults to the MIND.jl checkout's mod/ directory.  The mechanisms compiled into
libmindgpu.so this way are the cell mechanisms of that directory: SEClamp and VClamp,
which have no hand-written device code, and hh, pas, ExpSyn, Exp2Syn, IClamp and
AlphaSynapse, which also run through their hand-written paths (kinds 1-7) -- the generated
copies are selected by load_mod and are held bit-identical to the hand-written ones by the
parity tests.  NetStim (an artificial cell with its own self-event device code) and the
empty PatternStim placeholder are not emitted.  Extra MOD files are appended in order.
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from mind_b200.nmodl.library import library_header, read_sources  # noqa: E402

DEFAULT_DIR = "/root/reference/mod"
MECHANISMS = ["SEClamp", "VClamp", "hh", "pas", "ExpSyn", "Exp2Syn", "IClamp", "AlphaSynapse"]
OUTPUT = os.path.join(HERE, "generated_mechanisms.cuh")


def main(argv):
    mod_dir = argv[1] if len(argv) > 1 and os.path.isdir(argv[1]) else DEFAULT_DIR
    extra = [a for a in argv[1:] if a.endswith(".mod")]
    paths = [os.path.join(mod_dir, f"{name}.mod") for name in MECHANISMS] + extra
    text = library_header(read_sources(paths))
    with open(OUTPUT, "w") as f:
        f.write(text)
    print(OUTPUT)


if __name__ == "__main__":
    main(sys.argv)
