"""Copy the reference's golden input/outputs into gzip fixtures (run once).

The reference (takahashi-edalab/EUVlitho) ships one mask and the outputs of its
two drivers for it:

* ``cnn/intensity/abbe/mask.bin``   -> ref_mask.bin.gz   (2048x2048 bits, MSB first)
* ``cnn/intensity/abbe/emint.csv``  -> ref_emint.csv.gz  (512x512 Abbe intensity)
* ``cnn/intensity/m3d/inputxx.csv`` -> ref_inputxx.csv.gz (M3D parameters a0, ax, ay)
* ``cnn/intensity/m3d/inputlm.csv`` -> ref_inputlm.csv.gz (pupil orders l, m, xflag)

These are data, not source.  Usage: python tests/golden/make_golden.py [REFERENCE_ROOT]
"""
import gzip
import os
import sys

FILES = {
    "cnn/intensity/abbe/mask.bin": "ref_mask.bin.gz",
    "cnn/intensity/abbe/emint.csv": "ref_emint.csv.gz",
    "cnn/intensity/m3d/inputxx.csv": "ref_inputxx.csv.gz",
    "cnn/intensity/m3d/inputlm.csv": "ref_inputlm.csv.gz",
}


def main() -> int:
    from refroot import reference_root
    root = reference_root()
    here = os.path.dirname(os.path.abspath(__file__))
    for src, dst in FILES.items():
        with open(os.path.join(root, src), "rb") as fh:
            data = fh.read()
        with gzip.GzipFile(os.path.join(here, dst), "wb", mtime=0) as out:
            out.write(data)
        print(src, "->", dst, len(data), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
