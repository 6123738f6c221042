"""Location of the reference checkout that the oracle recipes read (read-only).

TEST INFRASTRUCTURE ONLY: used by the golden-vector scripts under
tests/golden/, the reference-caller tests and build(), never by the product.
Set NRLDPC_REFERENCE_ROOT to point elsewhere; the default is the checkout's
mount point in the build container.  The GPU box has no reference checkout:
everything that runs there uses the prebuilt oracle/_ref library and the
committed fixtures.
"""

import os

REFERENCE_ROOT = os.environ.get("NRLDPC_REFERENCE_ROOT", "/root/reference")


def reference_available() -> bool:
    return os.path.isfile(os.path.join(REFERENCE_ROOT, "c_lib", "nr_ldpc.h"))
