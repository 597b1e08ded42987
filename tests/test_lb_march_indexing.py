"""The index arithmetic of lb_march_kernel (csrc/lb_kernels.cu), restated on
the CPU: every global load and store in bounds, every shared-memory index in
range, every phase-2 pull from the ring finding the step-n value of the row
and column it needs, every output node computed exactly once, and the ring
rows that one group's phase 1 overwrites never read by the previous group's
phase 2 (the one barrier per group).  The chunking follows launch_march_t."""
import pytest

CX = [0, 1, 0, -1, 0, 1, -1, -1, 1]
CY = [0, 0, 1, 0, -1, 1, 1, -1, -1]


def chunk_height(ny, nx, R, waves, occ, nsm):
    """launch_march_t: H = kR - 2 for about `waves` waves of resident blocks"""
    nstrips = (nx + 31) // 32
    target = max(1, (waves * occ * nsm + nstrips // 2) // nstrips)
    h0 = (ny + target - 1) // target
    H = ((h0 + 2 + R - 1) // R) * R - 2
    return H, nstrips * ((ny + H - 1) // H)


def emulate(nx, ny, R, H, glo=False, ghi=False):
    RING, CW = 2 * R + 2, 34
    nstrips = (nx + 31) // 32
    nchunks = (ny + H - 1) // H
    covered = {}
    ylo, yhi = (-1 if glo else 0), (ny if ghi else ny - 1)
    for b in range(nstrips * nchunks):
        strip, chunk = b % nstrips, b // nstrips
        x0 = strip * 32
        ncols = min(32, nx - x0)
        ya = chunk * H
        Hc = min(H, ny - ya)
        assert Hc >= 1
        ring = {}  # (slot, ring column) -> (ly, x) of the step-n value held
        sfr = {}   # slot -> ly of F^{n+1}
        Q = (Hc + 2 + R - 1) // R
        prev_reads = set()  # (slot, column) read by the previous group's phase 2
        for q in range(Q):
            writes = set()
            for warp in range(R + 1):  # phase 1
                for lane in range(32):
                    if warp < R:
                        w, x, c, ok = warp, x0 + lane, lane + 1, lane < ncols
                    else:
                        right = lane >= R
                        w = lane - R if right else lane
                        c = ncols + 1 if right else 0
                        x = x0 + ncols if right else x0 - 1
                        x = x + nx if x < 0 else (x - nx if x >= nx else x)
                        ok = lane < 2 * R
                    ly = q * R + w
                    y = ya - 1 + ly
                    if not (ok and ly <= Hc + 1 and ylo <= y <= yhi):
                        continue
                    assert 0 <= x < nx and 0 <= c < CW
                    if 0 <= y < ny:
                        for k in range(9):  # the pulls (pull_node): in the domain or the wall row
                            js = y - CY[k]
                            assert 0 <= (x - CX[k]) % nx < nx
                            assert js < 0 or js >= ny or 0 <= js < ny
                    slot = ly % RING
                    assert 0 <= slot < RING
                    writes.add((slot, c))
                    ring[(slot, c)] = (ly, x)
                    if warp < R and 1 <= ly <= Hc:
                        assert 0 <= y < ny and x0 <= x < x0 + ncols
                        sfr[slot] = ly
            # the barrier of group q: this phase 1 must not overwrite what the
            # previous group's phase 2 reads (it may still run beside it)
            assert not (writes & prev_reads), (b, q)
            reads = set()
            for warp in range(R):  # phase 2
                for lane in range(32):
                    ly = q * R - 1 + warp
                    y = ya - 1 + ly
                    if not (lane < ncols and 1 <= ly <= Hc):
                        continue
                    x = x0 + lane
                    s0, sm, sp = ly % RING, (ly - 1) % RING, (ly + 1) % RING
                    for k in range(9):
                        js = y - CY[k]
                        if (js < 0 and not glo) or (js >= ny and not ghi):
                            key, want = (s0, lane + 1), (ly, x)  # bounce-back: own node
                        else:
                            sl = sm if CY[k] == 1 else (sp if CY[k] == -1 else s0)
                            cc = lane + 1 - CX[k]
                            assert 0 <= cc < CW
                            key, want = (sl, cc), (ly - CY[k], (x - CX[k]) % nx)
                        assert ring.get(key) == want, (b, q, warp, lane, k, ring.get(key), want)
                        reads.add(key)
                    assert sfr.get(s0) == ly
                    assert 0 <= y < ny
                    covered[(y, x)] = covered.get((y, x), 0) + 1
            prev_reads = reads
    assert len(covered) == nx * ny and set(covered.values()) == {1}


@pytest.mark.parametrize("nx,ny,R,H", [(64, 37, 8, 14), (200, 37, 8, 30), (96, 20, 4, 6), (48, 24, 16, 30),
                                       (40, 7, 6, 4), (16, 5, 8, 6), (128, 64, 8, 62), (33, 31, 4, 2)])
def test_march_indexing(nx, ny, R, H):
    emulate(nx, ny, R, H)


@pytest.mark.parametrize("glo,ghi", [(True, False), (False, True), (True, True)])
def test_march_indexing_slab_ghost_rows(glo, ghi):
    emulate(64, 13, 8, 14, glo, ghi)
    emulate(40, 9, 4, 6, glo, ghi)


@pytest.mark.parametrize("R,waves,occ", [(8, 8, 4), (4, 8, 8), (16, 8, 2), (6, 8, 5), (8, 3, 4), (8, 8, 3)])
@pytest.mark.parametrize("nx,ny", [(4096, 2048), (512, 256), (200, 37), (64, 24)])
def test_march_chunk_height(R, waves, occ, nx, ny):
    """whole groups per chunk, and a grid that covers the rows"""
    H, grid = chunk_height(ny, nx, R, waves, occ, 148)
    assert (H + 2) % R == 0 and H >= R - 2 and H >= 1
    nstrips = (nx + 31) // 32
    assert grid % nstrips == 0 and (grid // nstrips) * H >= ny > (grid // nstrips - 1) * H
