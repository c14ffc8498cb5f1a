"""ORACLE — test infrastructure only.

A CPU restatement of the reference's batched AFQMC walker step (bkesk/SAFIRE) used to check the
CUDA product path.  Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and only as the comparison
standard or as the timed CPU baseline.  The product package (``safire_b200``) never imports it.

Parity pins: the determinant / density-matrix / inverse functions are checked against the golden
values of the reference's tests/test_sdet_ops.cpp, the PHMSD two-body kernel against
tests/test_phmsd_components.cpp, and the RNG against libstdc++ (oracle/stdrng_ref.cpp).  The
Real3Index vbias / vHS / energy numbers have no stored golden values in the reference (its
molecular HDF5 fixtures carry no TEST_RESULTS group); the whole step is instead pinned by the
reference's seeded snapshot runs (tests/functional/snapshot_references of BH and N2): fed the
same host random streams, the oracle reproduces their reported energies to 1e-9
(tests/test_molecule_snapshots.py), on top of the internal-consistency tests in
tests/test_oracle_*.py.
"""
