"""CPU oracle of the SPH fluid-step path (test infrastructure only).

A C++17/OpenMP restatement of the reference's formulas (sph_oracle.hpp).
Only tests/, the smoke check and bench.py's CPU-baseline leg use it, as the
checker; the engine never does.
"""
