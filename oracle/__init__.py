"""The oracle: a CPU restatement of TorchCor's monodomain time step.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` may import this package, and only as the
checker (or as the timed CPU baseline).  The product path in ``torchcor_b200``
never imports it and has no CPU fallback.

``oracle.port`` restates, with plain PyTorch CPU ops in the reference's own
operation order, the functions of TorchCor 0.1.8 on the monodomain path
(mesh reading, conductivity, P1 assembly, Jacobi-PCG, stimuli, the three ionic
models and the ``Monodomain.solve`` loop).  Every function cites the reference
file:line it follows.

Parity pinning: the restatement is checked against golden vectors produced by
running the reference itself (``tests/golden/make_golden.py`` imports the
reference package and writes ``tests/golden/*.npz``); ``tests/test_oracle.py``
compares the two.
"""
