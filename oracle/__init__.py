"""CPU oracle for the ladder DGA hot path.

TEST INFRASTRUCTURE ONLY.  This package is the checker: a NumPy restatement of the upstream algorithm
(Julpe/DGAmore, pure Python + NumPy) for the bubble, the ladder Bethe-Salpeter solve, the vertex and kernel
assembly, the Schwinger-Dyson contraction, the lambda-correction and the Eliashberg matvec.  Each function
cites the upstream ``file:line`` it follows.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs of
``bench.py`` may import it.  The product package ``dgamore_b200`` never does; its GPU path fails loudly when
the CUDA library is missing.

Parity pins (see ``tests/test_oracle_pins.py``): the oracle reproduces the upstream's own golden fixtures
(``tests/test_data/end_2_end/gchi0_q_rank_0.npy``, ``gchi0_q_inv_rank_0.npy`` from ``g_dga.npy``; the
lambda-correction fixtures and values of ``tests/test_lambda_correction.py``; the BSE known-answer tests of
``tests/test_four_point.py:466-532``) and the outputs of the upstream code itself, run in FP64 on seeded
synthetic inputs by ``tests/golden/make_golden.py``.
"""
