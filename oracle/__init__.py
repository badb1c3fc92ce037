"""Oracle package (test infrastructure only): CPU restatements of the reference's
Hamiltonian-apply path used to check the CUDA product.  Imported only by tests/,
the smoke check and bench.py's cpu_baseline leg."""
