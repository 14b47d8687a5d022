"""The autotuner's cache key (host logic): the same batch and candidates
give the same key whatever the problem order; any change of GPU,
precision, size distribution or candidate list gives another."""
from cup2d_b200 import _lib as L
from cup2d_b200.poisson import tune_key


def test_tune_key():
    sizes = [50, 120, 3000, 800, 6000, 75]
    k = tune_key("NVIDIA B200", L.PREC_MIXED, sizes, (6, 8, 12), (0,))
    assert k == tune_key("NVIDIA B200", L.PREC_MIXED, list(reversed(sizes)), (6, 8, 12), (0,))
    others = [tune_key("NVIDIA H100", L.PREC_MIXED, sizes, (6, 8, 12), (0,)),
              tune_key("NVIDIA B200", L.PREC_FP64, sizes, (6, 8, 12), (0,)),
              tune_key("NVIDIA B200", L.PREC_MIXED, sizes + [20000], (6, 8, 12), (0,)),
              tune_key("NVIDIA B200", L.PREC_MIXED, sizes, (8, 12), (0,)),
              tune_key("NVIDIA B200", L.PREC_MIXED, sizes, (6, 8, 12), (0, 2))]
    assert len(set(others)) == len(others) and k not in others
