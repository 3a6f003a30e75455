"""The oracle: CPU restatement of the reference solver's hot path and a runner
for the reference's own code compiled from its sources (TEST INFRASTRUCTURE
ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference
legs of ``bench.py`` may import this package, and only as the checker or the
timed CPU baseline -- never as the product path.
"""
