"""mcq_qmc_pass_noalloc: the RQMC pass for callers that may not allocate GPU memory, checked
against the allocating entry point (mcq_qmc_pass_device) through the C ABI.

Runs last (file name) so that a stop-at-first-failure run has executed everything else
first; it sets the no-allocation scratch up itself and so passes in a fresh process too."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_pass(eng):
    import torch
    torch.cuda.set_device(0)
    m, p = eng.gbm(100.0, 0.03, 0.25, 1.0), eng.asian(100.0)
    R, n_steps = 8, 256
    stream = torch.cuda.Stream()
    ref = torch.zeros(2 * R, dtype=torch.float64, device="cuda")
    out = torch.zeros(2 * R, dtype=torch.float64, device="cuda")
    # two calls in a row with different salts / offsets: the shared scratch must not carry
    # anything from one call into the next
    for call, (salt, off, n) in enumerate([(42, 0, 20000), (97, 4096 + 5, 33333)]):
        eng.qmc_pass_noalloc(m, p, n_steps, out.data_ptr(), stream.cuda_stream, salt_base=salt, R=R, offset=off,
                             n_points=n)
        stream.synchronize()
        eng.qmc_pass_device(m, p, n_steps, ref.data_ptr(), stream.cuda_stream, salt_base=salt, R=R, offset=off,
                            n_points=n)
        stream.synchronize()
        a, b = out.cpu().numpy().reshape(R, 2), ref.cpu().numpy().reshape(R, 2)
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=0.0, err_msg=f"call {call}")
        assert np.all(a[:, 0] / n > 5) and np.all(a[:, 0] / n < 8)
    # a large pass (2^20 points x 32 replicas: the work split's full item count) fits the scratch
    R2 = 32
    ref2 = torch.zeros(2 * R2, dtype=torch.float64, device="cuda")
    out2 = torch.zeros(2 * R2, dtype=torch.float64, device="cuda")
    eng.qmc_pass_noalloc(m, p, n_steps, out2.data_ptr(), stream.cuda_stream, salt_base=42, R=R2, offset=0,
                         n_points=1 << 20)
    stream.synchronize()
    eng.qmc_pass_device(m, p, n_steps, ref2.data_ptr(), stream.cuda_stream, salt_base=42, R=R2, offset=0,
                        n_points=1 << 20)
    stream.synchronize()
    np.testing.assert_allclose(out2.cpu().numpy(), ref2.cpu().numpy(), rtol=1e-12, atol=0.0)
    # a call after set-up takes no device memory
    torch.cuda.synchronize()
    before = torch.cuda.mem_get_info()[0]
    eng.qmc_pass_noalloc(m, p, n_steps, out.data_ptr(), stream.cuda_stream, salt_base=5, R=R, offset=0,
                         n_points=1000)
    stream.synchronize()
    assert torch.cuda.mem_get_info()[0] == before


def test_noalloc_heston_and_limits(eng):
    import torch
    m, p = eng.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0), eng.lookback(0.2)
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    ref = torch.zeros(4, dtype=torch.float64, device="cuda")
    eng.qmc_pass_noalloc(m, p, 256, out.data_ptr(), 0, salt_base=7, R=2, offset=0, n_points=4096)
    eng.qmc_pass_device(m, p, 256, ref.data_ptr(), 0, salt_base=7, R=2, offset=0, n_points=4096)
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-12, atol=0.0)
    with pytest.raises(eng.MCQError) as e:   # 257 steps x 2 factors > 512 dimensions
        eng.qmc_pass_noalloc(m, p, 257, out.data_ptr(), 0, R=2, n_points=64)
    assert e.value.code == 4 and "512" in str(e.value)
    with pytest.raises(eng.MCQError) as e:
        eng.qmc_pass_noalloc(eng.gbm(), p, 64, out.data_ptr(), 0, R=33, n_points=64)
    assert e.value.code == 4


@pytest.mark.parametrize("model,pay,n_steps", [
    ("dupire", "eur", 64),      # parametric Dupire, plain pass
    ("dupire", "asian", 300),   # long paths: the allocating entry point may take its assisted form
    ("gbm", "asian", 8),        # 8 normals a path: the packed pass with whole-tile work items
    ("heston", "eur", 4),       # 2 factors x 4 steps = 8 normals: packed as well
    ("gbm", "eur", 16),         # the packed limit
])
def test_noalloc_models_and_short_paths(eng, model, pay, n_steps):
    """Parametric Dupire and paths of at most 16 normals (where the allocating pass switches to
    its packed kernel) give the allocating entry point's sums bit for bit, twice in a row."""
    import torch
    m = {"gbm": lambda: eng.gbm(100.0, 0.03, 0.25, 1.0),
         "dupire": lambda: eng.dupire(100.0, 0.05, 0.2, 0.5, 0.7, 1.0),
         "heston": lambda: eng.heston(100.0, 0.02, 2.0, 0.04, 0.3, -0.7, 0.04, 1.0)}[model]()
    p = eng.european(100.0, 0.05, 1.0) if pay == "eur" else eng.asian(100.0)
    R = 4
    out = torch.zeros(2 * R, dtype=torch.float64, device="cuda")
    ref = torch.zeros(2 * R, dtype=torch.float64, device="cuda")
    for salt, off, n in ((11, 0, 40000), (12, 777, 5000)):
        eng.qmc_pass_noalloc(m, p, n_steps, out.data_ptr(), 0, salt_base=salt, R=R, offset=off, n_points=n)
        eng.qmc_pass_device(m, p, n_steps, ref.data_ptr(), 0, salt_base=salt, R=R, offset=off, n_points=n)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.array_equal(a, b), (model, n_steps, salt, a, b)
        assert np.all(np.isfinite(a)) and np.all(a[0::2] > 0)
