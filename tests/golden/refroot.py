"""Where the fixture scripts find the reference checkout.

The first command-line argument, else the environment variable
EUVLITHO_REFERENCE, else a directory named ``reference`` beside this
repository.  The scripts read the reference only to make fixtures; nothing in
the tests reads it."""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def reference_root() -> str:
    if len(sys.argv) > 1:
        root = sys.argv[1]
    else:
        root = os.environ.get("EUVLITHO_REFERENCE") or os.path.join(os.path.dirname(REPO),
                                                                     "reference")
    if not os.path.isdir(os.path.join(root, "cnn")):
        raise SystemExit("reference checkout not found at %r: pass it as the first argument "
                         "or set EUVLITHO_REFERENCE" % root)
    return root
