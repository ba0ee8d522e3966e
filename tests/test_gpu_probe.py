"""The FP32 FMA rate probe (mdb_fp32_fma_rate), the roofline denominator of the
mixed cluster-pair force kernels: a positive rate no farther than 25 % from
the figure of 128 FP32 lanes x 2 flops per SM and clock at the device's
current maximum clock, and no faster than the FP32 work it counts allows."""
import pytest

import mdb

pytestmark = pytest.mark.gpu


def test_fp32_fma_rate_is_plausible():
    torch = pytest.importorskip("torch")
    p = torch.cuda.get_device_properties(0)
    rate = mdb.fp32_fma_rate(0)
    clock_hz = torch.cuda.clock_rate(0) * 1e6 if hasattr(torch.cuda, "clock_rate") else 1.965e9
    nominal = p.multi_processor_count * 128 * 2 * clock_hz
    assert 0.75 * nominal <= rate <= 1.25 * nominal, (rate, nominal)
