"""Measurement drivers behind bench.py's sections (and runnable on their own,
``python -m benchmarks.<name> ...``): the learned-cache time-to-RMSE
comparison, the multi-scene probe batches, the 4 M-triangle city frame, the
cache consumers and the probe placement. They use the nan_b200 package and
are not part of it."""
