"""CPU oracle for the equirectangular RF splatting path.

TEST INFRASTRUCTURE ONLY: the tests, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` use it as the checker.  The product path never
imports it and has no CPU fallback.
"""
