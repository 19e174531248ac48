"""Device building blocks of the top level (GPU): the stable LSD radix sort of 64-bit grid keys used by
the dilation, against torch.sort."""
import ctypes as C

import pytest

from sincfeyn_b200 import sq

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('n,nbits', [(1, 8), (1000, 20), (1 << 20, 44), (3_000_001, 41)])
def test_radix_sort_matches_torch(n, nbits):
    import torch
    g = torch.Generator(device='cpu').manual_seed(n)
    keys = torch.randint(1, 1 << nbits, (n,), generator=g, dtype=torch.int64)
    d = keys.cuda()
    L = sq.lib()
    L.sqb_radix_sort_u64.argtypes = [C.c_void_p, C.c_long, C.c_int, C.c_void_p]
    torch.cuda.synchronize()
    assert L.sqb_radix_sort_u64(d.data_ptr(), n, nbits, None) == 0
    torch.cuda.synchronize()
    assert torch.equal(d.cpu(), torch.sort(keys).values)
