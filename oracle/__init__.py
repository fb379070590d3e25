"""The oracle: TEST INFRASTRUCTURE ONLY.

CPU restatements of the reference's projector path (``cbct_oracle.c``), the
reference's own CPU C compiled from its sources (``_ref/libcbct_ref.so``, built
by ``oracle/Makefile`` where the reference checkout exists), and numpy
restatements of the MATLAB callers.  Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline legs may import this package; the product
package ``ctsim_b200`` never does.
"""
