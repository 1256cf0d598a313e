"""The cell-crossing rule of the CPU oracle (no GPU needed).

move_mode 0 is the reference's push (src/cuda_Move.cu:227-255): one wrap of
the in-cell offset per step, so a particle faster than one cell per step keeps
an offset outside [0, 1).  move_mode 1 crosses cell by cell, applying the
boundary rule of every cell entered (src/cuda_Sortboundary.cu:70-256), until
the offset is inside a cell.  These tests pin the two rules on the oracle; the
GPU kernels are compared with the oracle bit for bit in test_gpu_ops.py.
"""
import numpy as np
import pytest

import hpic
import oracle
from hpic.decks import block_deck, ccp_deck


def _oracle(move_mode, cells_per_step=None, every=3, deck=None):
    deck = deck or ccp_deck(65, 33, 0.02, 0.01, ppc=8)
    S = hpic.Setup(deck, seed=11, field_mode=2, move_mode=move_mode, gas_temp_mode=1)
    o = oracle.from_setup(S, 32, field_mode=2)
    if cells_per_step is not None:
        info = S.info
        counts, (x, y, vx, vy, vz) = o.particles(0)
        k = np.arange(x.size)
        sel = k % every == 0
        sign = np.where((k // every) % 2 == 0, 1, -1).astype(np.float32)
        vcx = np.float32(cells_per_step * info.dx / info.dt)
        vcy = np.float32(0.5 * cells_per_step * info.dy / info.dt)
        vx = np.where(sel, sign * vcx, vx).astype(np.float32)
        vy = np.where(sel, -sign * vcy, vy).astype(np.float32)
        o.set_particles(0, counts, x, y, vx, vy, vz)
    o.DepositBasic()
    return S, o


def _push(o, t=1):
    o.Field(t)
    o.Move()


@pytest.mark.parametrize("cells", [2.6, 7.3])
def test_walk_keeps_offsets_inside_a_cell(cells):
    S, o = _oracle(1, cells)
    _push(o)
    counts, _, codes = o.movers(0)
    assert (codes == 14).sum() > 0, "no mover beyond the 3x3 neighbourhood"
    assert set(np.unique(codes)) <= set(range(9)) | {14, 15}
    o.SortBoundary()
    _, (x, y, vx, vy, vz) = o.particles(0)
    assert x.min() >= 0 and x.max() < 1 and y.min() >= 0 and y.max() < 1
    assert not o.walk_bound_hit()


def test_reference_wrap_keeps_one_crossing():
    S, o = _oracle(0, 2.6)
    _push(o)
    _, _, codes = o.movers(0)
    # one crossing: every destination lies in the 3x3 neighbourhood
    assert set(np.unique(codes)) <= set(range(9)) | {15}
    o.SortBoundary()
    _, (x, *_r) = o.particles(0)
    assert x.max() >= 1 or x.min() < 0


def test_walk_conserves_particles_and_tallies_absorption():
    """Every particle either stays or is absorbed; the block deck's
    conductors (StructureIndex codes >= 100) count what they absorb, the
    plate deck's electrode rows (ghost code -1) absorb without a count, as in
    the reference (src/cuda_Sortboundary.cu:70-256)."""
    for deck, counted in ((block_deck(), True), (None, False)):
        S, o = _oracle(1, 7.3, deck=deck)
        n0 = [o.particles(s)[1][0].size for s in range(S.info.nsp)]
        _push(o)
        absorbed = []
        for s in range(S.info.nsp):
            _, _, codes = o.movers(s)
            absorbed.append(int((codes == 15).sum()))
        o.SortBoundary()
        cc = o.counters()[0][: S.info.nsp * S.info.cond_numr].reshape(S.info.nsp, S.info.cond_numr)
        for s in range(S.info.nsp):
            assert o.particles(s)[1][0].size == n0[s] - absorbed[s]
            assert int(cc[s].sum()) <= absorbed[s]
        assert absorbed[0] > 0
        assert (int(cc[0].sum()) > 0) == counted


def test_walk_reflection_mirrors_the_side_walls():
    """A particle sent left across the x = 0 Neumann wall comes back with its
    x velocity reversed and its distance to the wall mirrored."""
    S, o = _oracle(1)
    info = S.info
    C = info.Csize
    counts = np.zeros(C, np.int32)
    j = info.ncy // 2
    counts[0 * info.ncy + j] = 1  # cell (0, j)
    x = np.array([0.25], np.float32)
    y = np.array([0.5], np.float32)
    vcx = np.float32(-2.5 * info.dx / info.dt)  # 2.5 cells to the left
    o.set_particles(0, counts, x, y, np.array([vcx], np.float32), np.zeros(1, np.float32),
                    np.zeros(1, np.float32))
    o.set_grid("EX", np.zeros(info.Gsize, np.float32))
    o.set_grid("EY", np.zeros(info.Gsize, np.float32))
    o.Move()
    o.SortBoundary()
    cnt, (px, py, pvx, _vy, _vz) = o.particles(0)
    # x = 0.25 - 2.5 = -2.25 cells -> mirrored to +2.25 cells: cell 2, offset 0.25
    assert cnt[2 * info.ncy + j] == 1 and px.size == 1
    assert abs(px[0] - 0.25) < 1e-6 and pvx[0] == -vcx
