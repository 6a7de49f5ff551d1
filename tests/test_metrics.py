from gvdb2 import metrics


def test_stage_bytes_formula():
    s = metrics.stage_bytes(N=1000, B=10, U=20, C=4, Cw=4, G=3, T=1000, R3=512, CL=4096)
    assert s["topology"] == 12 * 1000 + 4 * 1000 + 8 * 20 + 64 * 20 + 4096
    assert s["binning"] == 8000
    assert s["scatter"] == 12000 + 16000 + 4000 + 4 * 4 * 10 * 1000
    assert s["apron"] == 2 * 4 * 4 * 10 * 488
    assert s["gather"] == 12000 + 4000 + 12000 + 4 * 3 * 10 * 1000
    assert metrics.step_bytes(N=1000, B=10, U=20, C=4, Cw=4, G=3, T=1000, R3=512, CL=4096) == sum(s.values())


def test_adjoint_bytes():
    assert metrics.adjoint_bytes(N=10, B=2, C=1, Cw=1, T=1000) == 4 * 2 * 1000 + 16 * 10
