"""storm_b200 -- B200-native FVT time step for SToRM (scharlton2/storm).

The product is the C-ABI library ``libstorm_fvt.so`` (include/storm_fvt.h) built from
``storm_b200/csrc``; :mod:`storm_b200.fvt` is its Python host binding and
:mod:`storm_b200.scenarios` the seeded synthetic workloads.
"""
