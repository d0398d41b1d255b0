"""Location of the reference checkout whose sources the harness recipes compile where
they lie (test infrastructure): $CUOPO3D_REFERENCE, else the default checkout path."""
import os

DEFAULT_REFERENCE_ROOT = "/root/reference"


def reference_root():
    return os.environ.get("CUOPO3D_REFERENCE", DEFAULT_REFERENCE_ROOT)
