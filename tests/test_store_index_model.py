"""CPU model of the encoder's chunk store (store_shifted in
sleek_b200/csrc/sleek_device.cuh): the chunk's bytes, staged at a 16-byte aligned
shared-memory address, go to an arbitrary global byte address as 16-byte stores,
each funnel-shifted from two aligned staged granules, consecutive threads on
consecutive granules and two granules in flight per thread, and byte stores by the
first warp for the two granules shared with the neighbouring chunks.  The model
repeats the kernel's index arithmetic thread by thread (the producer warp's 32
threads, which store the chunks as their stages are refilled, and the compute
warps' 256 threads, which store the last chunks) and checks, for every byte misalignment and chunk lengths from 1 byte to a
full raw chunk: every destination byte is written exactly once, nothing outside the
chunk's bytes is written, and every staged read stays inside the stage."""
import pytest

STAGE_BYTES = 16384 + 64


def model(sft, ln, NT):
    a0 = 64  # a 16-byte aligned base
    dst = a0 + sft
    nunits = (sft + ln + 15) >> 4
    jf = 1 if sft else 0
    jl = (sft + ln) >> 4
    written, reads = {}, set()

    def wr(b):
        written[b] = written.get(b, 0) + 1

    def granule(j):
        reads.update((j - 1, j) if sft else (j,))
        for b in range(16):
            wr(a0 + 16 * j + b)

    for t in range(NT):
        if sft == 0:
            for j in range(t, jl, NT):
                granule(j)
        else:
            for j in range(jf + t, jl, 2 * NT):
                granule(j)
                if j + NT < jl:
                    granule(j + NT)
        if t >= 32:
            continue
        e = -1
        if t < 16:
            if sft != 0:
                e = 0
        else:
            last = nunits - 1
            if last >= jl and not (last == 0 and sft != 0):
                e = last
        if e >= 0:
            r = 16 * e - sft + (t & 15)
            if 0 <= r < ln:
                wr(a0 + 16 * e + (t & 15))
    return dst, written, reads


LENGTHS = list(range(1, 200)) + [255, 256, 257, 511, 512, 513, 1000, 4097, 8000, 16383 - 17, 16383, 16384]


@pytest.mark.parametrize("nt", (32, 256))
@pytest.mark.parametrize("sft", range(16))
def test_store_writes_every_byte_once_and_nothing_else(sft, nt):
    for ln in LENGTHS:
        dst, written, reads = model(sft, ln, nt)
        assert all(written.get(b, 0) == 1 for b in range(dst, dst + ln)), (sft, ln)
        assert all(dst <= b < dst + ln for b in written), (sft, ln)
        assert all(0 <= g and 16 * (g + 1) <= STAGE_BYTES for g in reads), (sft, ln)
