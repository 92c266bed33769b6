"""B200-native engine for the rank-adaptive BUG step of madhavmen/BondUpdateGalerkin.

``cbe_bug_step`` (``step.py``) is the drop-in for ``cbe_bug_step!``
(``src/BUG/TimeEvolution/bug_step.jl:17-513``); its tensors live in HBM as engine handles
(``tensor.py``) and every contraction, factorisation and reduction runs in ``libbug_b200.so``.
"""

__version__ = "0.1.0"
