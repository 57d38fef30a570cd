"""Copy the reference's own positions fixture into tests/golden.

The reference ships one realistic-geometry input for this path:
relearn/input/positions.txt (51,842 neurons with brain-area labels, the
simulation box in its "# Minimum/Maximum" header lines), in the format that
NeuronIO::read_neuron_positions_and_signals (io/NeuronIO.cpp:229-300) reads.
The GPU tests run it through the library's positions readers, and the
reference tree is not available where they run, so the file is kept here
byte for byte, xz-compressed, with its SHA-256 beside it.  Run from the
repository root of a checkout that has the reference at REFERENCE (default
/root/reference):

    python tests/golden/make_reference_positions.py
"""
import hashlib
import lzma
import os
import sys

OUT = os.path.dirname(os.path.abspath(__file__))
NAME = "reference_positions.txt"


def main():
    ref = os.environ.get("REFERENCE", "/root/reference")
    src = os.path.join(ref, "relearn", "input", "positions.txt")
    with open(src, "rb") as f:
        data = f.read()
    with lzma.open(os.path.join(OUT, NAME + ".xz"), "wb", preset=9 | lzma.PRESET_EXTREME) as f:
        f.write(data)
    with open(os.path.join(OUT, NAME + ".sha256"), "w") as f:
        f.write(hashlib.sha256(data).hexdigest() + "  " + NAME + "\n")
    print(f"{src}: {len(data)} bytes -> {NAME}.xz", file=sys.stderr)


if __name__ == "__main__":
    main()
