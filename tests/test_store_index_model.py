"""CPU model of the encoder's chunk store (store_shifted in
sleek_b200/csrc/sleek_device.cuh): the chunk's bytes, staged at a 16-byte aligned
shared-memory address, go to an arbitrary global byte address as 32-byte aligned
pair stores (three staged granules each), at most two single 16-byte granules, and
byte stores for the two granules shared with the neighbouring chunks.  The model
repeats the kernel's index arithmetic thread by thread (the compute warps' 256
threads, and one warp) and checks, for every byte misalignment, both pair parities
and chunk lengths from 1 byte to a full raw chunk: every destination byte is written
exactly once, nothing outside the chunk's bytes is written, every pair store is
32-byte aligned, and every staged read stays inside the stage."""
import pytest

STAGE_BYTES = 16384 + 64


def model(sft, par, ln, nt):
    a0 = 16 * (2 + par)  # a 16-byte aligned base whose granule index has parity `par`
    dst = a0 + sft
    nunits = (sft + ln + 15) >> 4
    jf = 1 if sft else 0
    jl = (sft + ln) >> 4
    written, reads, pairs = {}, set(), []

    def wr(b):
        written[b] = written.get(b, 0) + 1

    jp = jf + ((jf + par) & 1)
    np_ = (jl - jp) >> 1 if jl - jp >= 0 else 0
    for lane in range(nt):
        for k in range(lane, np_, nt):
            j = jp + 2 * k
            pairs.append(a0 + 16 * j)
            reads.update((j - 1, j, j + 1) if sft else (j, j + 1))
            for b in range(32):
                wr(a0 + 16 * j + b)
        j = -1
        if lane == 0 and jp > jf and jf < jl:
            j = jf
        if lane == 1 and jp + 2 * np_ < jl:
            j = jp + 2 * np_
        if j >= 0:
            reads.update((j - 1, j) if sft else (j,))
            for b in range(16):
                wr(a0 + 16 * j + b)
        if lane >= 32:
            continue
        e = -1
        if lane < 16:
            if sft != 0:
                e = 0
        else:
            last = nunits - 1
            if last >= jl and not (last == 0 and sft != 0):
                e = last
        if e >= 0:
            r = 16 * e - sft + (lane & 15)
            if 0 <= r < ln:
                wr(a0 + 16 * e + (lane & 15))
    return dst, written, reads, pairs


LENGTHS = list(range(1, 200)) + [255, 256, 257, 511, 512, 513, 1000, 4097, 8000, 16383 - 17, 16383, 16384]


@pytest.mark.parametrize("nt", [32, 256])
@pytest.mark.parametrize("sft", range(16))
def test_store_writes_every_byte_once_and_nothing_else(sft, nt):
    for par in (0, 1):
        for ln in LENGTHS:
            dst, written, reads, pairs = model(sft, par, ln, nt)
            assert all(written.get(b, 0) == 1 for b in range(dst, dst + ln)), (sft, par, ln)
            assert all(dst <= b < dst + ln for b in written), (sft, par, ln)
            assert all(p % 32 == 0 for p in pairs), (sft, par, ln)
            # staged granules read: inside the stage and inside the chunk's granules
            assert all(0 <= g and 16 * (g + 1) <= STAGE_BYTES and 16 * g < sft + ln for g in reads), (sft, par, ln)
