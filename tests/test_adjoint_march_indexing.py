"""The index arithmetic of adjoint_march_kernel (csrc/adjoint_kernels.cu),
restated on the CPU: every load and store in bounds, every ring read finds
the row and column it needs, written in the same run of the block, every
phase-2 node computed exactly once, and the ring rows one group's phase 1
writes are not read by the previous group's phase 2 (the one barrier per
group).  The grid and chunking follow launch_march_o."""
import pytest

CX = [0, 1, 0, -1, 0, 1, -1, -1, 1]
CY = [0, 0, 1, 0, -1, 1, 1, -1, -1]


def chunking(nx, ny, RB, slots, waves):
    ngroups = (ny + RB - 1) // RB
    nstrips = (nx + 31) // 32
    target = max(1, slots * waves // nstrips)  # chunks per strip
    chunk = (ngroups + target - 1) // target
    nchunks = (ngroups + chunk - 1) // chunk
    return ngroups, nstrips, chunk, nstrips * nchunks


def emulate(nx, ny, RB, slots, waves):
    HX, S, NT = 34, 2 * RB + 2, 34 * RB
    ngroups, nstrips, chunk, grid = chunking(nx, ny, RB, slots, waves)
    covered = {}
    for b in range(grid):
        g0 = (b // nstrips) * chunk
        if g0 >= ngroups:
            continue
        ub = (b % nstrips) * ngroups + g0
        ue = ub + min(chunk, ngroups - g0)
        ring, run, prev_reads = {}, 0, set()
        st = (ub, True)
        while True:
            u, pro = st
            s, r = u // ngroups, (u % ngroups) * RB
            x0 = 32 * s
            if pro and u != ub:
                run, prev_reads = run + 1, set()  # the barrier before a prologue inside a run
            writes = set()
            for t in range(NT):  # phase 1
                hx, hy = t % HX, t // HX
                j1 = (r - RB if pro else r) + 1 + hy
                xh = x0 - 1 + hx
                xh = nx - 1 if xh == -1 else (0 if xh == nx else xh)
                if not (0 <= j1 < ny and xh < nx and (not pro or hy >= RB - 2)):
                    continue
                for k in range(9):  # the pulls of the forward state
                    xs = (xh - CX[k]) % nx
                    js = j1 - CY[k]
                    if not 0 <= js < ny:
                        js, xs = j1, xh
                    assert 0 <= js < ny and 0 <= xs < nx
                writes.add(j1 % S)
                ring[(j1 % S, hx)] = (j1, xh, run)
            assert not writes & prev_reads
            if not pro:
                reads = set()
                for t in range(32 * RB):  # phase 2
                    px, py = t % 32, t // 32
                    j2, x2 = r + py, x0 + px
                    if not (j2 < ny and x2 < nx):
                        continue
                    covered[(j2, x2)] = covered.get((j2, x2), 0) + 1
                    c = px + 1
                    for m in range(9):
                        sj = j2 + CY[m]
                        if 0 <= sj < ny:
                            assert ring.get((sj % S, c + CX[m])) == (sj, (x2 + CX[m]) % nx, run)
                            reads.add(sj % S)
                        else:
                            assert ring.get((j2 % S, c)) == (j2, x2, run)
                    for k in range(9):  # the pushes
                        xs = (x2 - CX[k]) % nx
                        js = j2 - CY[k]
                        if not 0 <= js < ny:
                            js, xs = j2, x2
                        assert 0 <= js < ny and 0 <= xs < nx
                    reads.add(j2 % S)
                prev_reads = reads
            st = (u, False) if pro else (u + 1, (u + 1) % ngroups == 0)
            if st[0] >= ue:
                break
    assert all(covered.get((j, x)) == 1 for j in range(ny) for x in range(nx))


@pytest.mark.parametrize("nx,ny", [(48, 24), (40, 13), (16, 8), (33, 7), (96, 31), (256, 96)])
@pytest.mark.parametrize("RB", [3, 4, 5, 6, 7])
def test_marching_kernel_indexing(nx, ny, RB):
    for slots, waves in [(296, 1), (296, 2), (148, 2), (3, 1), (1, 1)]:
        emulate(nx, ny, RB, slots, waves)
