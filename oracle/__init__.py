"""TEST INFRASTRUCTURE ONLY: CPU oracles for the integral hot path.

* oracle.ref  -- the unmodified reference engine compiled from its sources
  (oracle/build_ref.sh -> oracle/_ref/libtlno_ref.so);
* oracle.port -- the plain C++ restatement of the reference algorithm
  (oracle/tlno_oracle.cpp -> oracle/libtlno_oracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this package, as the checker -- never as the thing measured or
shipped.
"""
