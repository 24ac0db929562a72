"""tf_scan_exclusive_i32_noalloc, the scan for callers that cannot allocate
device memory: called through the C ABI it must give exactly the result of
the allocating tf_scan_exclusive_i32 (integer sums: tolerance zero), on two
calls in a row whose sizes differ, so that what the first call leaves in the
shared scratch array cannot leak into the second.  Collected last on
purpose, and self-contained, so it passes alone in a fresh process too."""
import ctypes

import pytest
import torch

import thermofem_b200 as tf

pytestmark = pytest.mark.gpu


def noalloc_scan(stream, x, out):
    return tf.lib().tf_scan_exclusive_i32_noalloc(ctypes.c_void_p(stream), x.numel(), ctypes.c_void_p(x.data_ptr()),
                                                  ctypes.c_void_p(out.data_ptr()))


# (70_000_000, 4_194_305): a three-level scan, then a two-level one whose
# first-level sums overlap what the first call left in the second-level region
@pytest.mark.parametrize("sizes", [(5_000_003, 1_777), (2_048, 70_000_000), (4_194_305, 4_194_305),
                                   (70_000_000, 4_194_305)])
def test_noalloc_scan_matches_allocating_scan_twice(ctx, sizes):
    stream = ctx.stream.cuda_stream
    for call, n in enumerate(sizes):
        g = torch.Generator(device="cuda").manual_seed(100 + call)
        x = torch.randint(0, 7, (n,), dtype=torch.int32, device="cuda", generator=g)
        want = tf.scan_exclusive(x, ctx=ctx)
        got = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        assert noalloc_scan(stream, x, got) == tf.OK, tf.lib().tf_last_error()
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}: n={n}"


def test_noalloc_scan_in_place_and_limits(ctx):
    stream = ctx.stream.cuda_stream
    x = torch.arange(10_000, dtype=torch.int32, device="cuda") % 5
    want = tf.scan_exclusive(x, ctx=ctx)
    torch.cuda.synchronize()
    assert noalloc_scan(stream, x, x) == tf.OK
    torch.cuda.synchronize()
    assert torch.equal(x, want)
    big = (1 << 27) + 1
    status = tf.lib().tf_scan_exclusive_i32_noalloc(ctypes.c_void_p(stream), big, ctypes.c_void_p(x.data_ptr()),
                                                    ctypes.c_void_p(x.data_ptr()))
    assert status == tf.ERR_LENGTH
    assert b"limit" in tf.lib().tf_last_error()
    empty = torch.empty(0, dtype=torch.int32, device="cuda")
    assert noalloc_scan(stream, empty, empty) == tf.OK


def test_noalloc_scan_allocates_nothing_after_its_first_call(ctx):
    # The first call on a device may load the module (lazy loading); after
    # it, scans of several sizes leave the device's free memory and torch's
    # caching pool exactly as they were: no call kept any device memory.
    stream = ctx.stream.cuda_stream
    xs = [torch.randint(0, 9, (n,), dtype=torch.int32, device="cuda") for n in (1_000, 3_000_000, 70_000_000)]
    outs = [torch.empty_like(x) for x in xs]
    torch.cuda.synchronize()
    # warm-up with the three-level size, which launches both of its kernels
    # (CUDA may also load each kernel lazily on its first launch)
    assert noalloc_scan(stream, xs[2], outs[2]) == tf.OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    pool0 = torch.cuda.memory_reserved()
    for _ in range(2):
        for x, out in zip(xs, outs):
            assert noalloc_scan(stream, x, out) == tf.OK, tf.lib().tf_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_reserved() == pool0
    for x, out in zip(xs, outs):
        assert torch.equal(out, tf.scan_exclusive(x, ctx=ctx))
