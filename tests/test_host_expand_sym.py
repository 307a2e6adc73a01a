"""CPU check of the index arithmetic of the expansion's symmetric plane writer
(``pipeline.cu::write_plane_sym``): a mirror of its mapping of threads to plane elements, run for
every N up to 69 and a few larger ones, must write every element of the N x N plane exactly once,
each from the table entry of (c, d) or of (d, c) (the same pair function)."""
import pytest


def plane_writes(n, nthreads):
    nw = nthreads // 32
    nq = (n + 3) >> 2
    written = {}

    def put(pos, src):
        assert pos not in written, (n, pos)
        written[pos] = src
    for t in range(nq * 16):  # the quads' 4 x 4 diagonal blocks
        c, d = 4 * (t >> 4) + ((t >> 2) & 3), 4 * (t >> 4) + (t & 3)
        if c < n and d < n:
            put((c, d), (c, d))
    for warp in range(nw):  # units (quad, 32-column chunk) round robin over the warps
        k = first = 0
        u = warp
        while True:
            while k < nq:
                chunks = (max(0, n - 4 * k - 4) + 31) >> 5
                if u < first + chunks:
                    break
                first += chunks
                k += 1
            if k >= nq:
                break
            c0 = 4 * k
            for lane in range(32):
                d = c0 + 4 + 32 * (u - first) + lane
                if d >= n:
                    continue
                assert c0 + 3 < n  # the transposed run of four is whole
                for i in range(4):
                    put((c0 + i, d), (c0 + i, d))
                    put((d, c0 + i), (c0 + i, d))
            u += nw
    return written


@pytest.mark.parametrize("nthreads", [512, 256])
def test_symmetric_plane_writer_covers_each_element_once(nthreads):
    for n in list(range(1, 70)) + [120, 121, 255, 420]:
        w = plane_writes(n, nthreads)
        assert len(w) == n * n
        assert all(src in ((c, d), (d, c)) for (c, d), src in w.items())
