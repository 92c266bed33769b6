"""B200-native engine for the rank-adaptive BUG step of madhavmen/BondUpdateGalerkin.

``native.cbe_bug_step`` (exported by ``api``) is the drop-in for ``cbe_bug_step!``
(``src/BUG/TimeEvolution/bug_step.jl:17-513``): the whole step runs in ``libbug_b200.so`` (the
sweep logic in C++, ``csrc/step.cu``; every contraction, factorisation and reduction as sm_100a
kernels) on tensors that live in HBM as engine handles (``tensor.py``).
"""

__version__ = "0.2.0"
