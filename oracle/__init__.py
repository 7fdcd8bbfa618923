"""The oracle: CPU restatement of the reference's hydro force path (FP64) and
the reference's own compiled CPU functors.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs, as the checker; the product
(weaklycompressiblesph_b200) never imports it.

* ``liboracle.so``        oracle/wcsph_oracle.c, the restatement (built by oracle/Makefile)
* ``_ref/libwcsph_ref.so`` oracle/ref_oracle.cpp compiled against the reference's
                          unmodified headers (built only where the reference
                          source tree exists; it then travels as a binary)

Parity of the restatement is pinned against the reference build by
tests/test_oracle_pin.py and against committed vectors in tests/golden/.
"""
from .bind import *  # noqa: F401,F403
