"""Test infrastructure: CPU oracles of the FVM kinetic update (numpy FP64
restatement in bolt_oracle.py; C/OpenMP FP64 restatement of the fields-off
path in bolt_oracle_c.c).  Only tests, the smoke check and bench.py's CPU
legs use this package; the product (bolt_b200) never imports it."""
