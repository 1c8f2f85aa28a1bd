"""Oracle: CPU restatement of the reference's parameterization, validation and
metrics arithmetic (numpy / scipy, FP64).

TEST INFRASTRUCTURE ONLY. Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import anything under ``oracle/``, and
only as the checker or as the timed CPU baseline. The product package
(``ultimate_uv_artist_b200``) never imports it and has no CPU fallback.

Each function cites the reference file:line it restates (paths inside the
Ultimate UV Artist project). The restatement is pinned against the reference
itself by ``tests/golden/make_golden.py`` (fixtures generated by importing the
reference) and ``tests/test_oracle_golden.py``.
"""
