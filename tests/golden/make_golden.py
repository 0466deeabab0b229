"""Regenerate the golden fixtures of this directory from a SemiImplicitFV
checkout, given as the first argument or by SIFV_REFERENCE_DIR.  The two CSV
files are the reference's published error tables for 1D periodic advection
(examples/1D_advection/explicitError.csv, semiImplicitError.csv), copied
verbatim as data so the tests can run where the reference is absent."""
import os
import shutil
import sys

src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIFV_REFERENCE_DIR")
if not src:
    sys.exit("usage: make_golden.py <SemiImplicitFV checkout>  (or set SIFV_REFERENCE_DIR)")
here = os.path.dirname(os.path.abspath(__file__))
for a, b in (("explicitError.csv", "advection_explicit_error.csv"),
             ("semiImplicitError.csv", "advection_semi_implicit_error.csv")):
    shutil.copyfile(os.path.join(src, "examples", "1D_advection", a), os.path.join(here, b))
    print("wrote", b)
