"""Suffix array of ONE text spread over several GPUs, one process per GPU.

The reference builds a single suffix array over p MPI ranks
(PDCX::compute_sa, lightweight_dcx/src/pdcx/pdcx.hpp:529-941):

  * the text is cut into p consecutive blocks (mpi/io.hpp:33-65) and each rank
    reads the first characters of its right neighbour's block so that windows
    crossing the boundary can be formed (shift_entries_left, mpi/shift.hpp:50-56);
  * every phase materialises records and sorts them with a distributed sample
    sort: local sort, splitters from a regular sample gathered on all ranks,
    bucket counts, an alltoallv of the records and a local merge
    (sorters/sample_sort.hpp:36-171, mpi/alltoall.hpp:106-137);
  * lexicographic names are offset by the number of distinct windows on lower
    ranks (compute_ranks.hpp:89-134), and a text whose names are not distinct
    recurses on the names in (i mod X, i div X) order (pdcx.hpp:146-212,
    compute_ranks.hpp:49-56), the ranks travelling back to the positions
    (map_back, pdcx.hpp:83-94);
  * the merge phase orders suffixes by their first characters and, where those
    tie, by the difference-cover comparator on the ranks of the following
    samples (merge_samples.hpp:87-109, 181-188).

This module keeps that structure over torch.distributed (NCCL between GPUs;
any backend with all_to_all_single).  One window sort of all suffixes serves
phase 1 (restricted to the samples) and phase 4, as in the single-GPU build.
Its local steps run on the rank's GPU: the sorts are the library's onesweep
radix passes (dcx_sort_u32), the recursion below `base_threshold` characters
is the single-GPU build of a 32-bit string (dcx_build_sa_u32) on rank 0, and
the rest are elementwise tensor operations on the rank's device.  The local
steps come from a `LocalOps` object: DeviceOps for GPUs.  There is no CPU
path in the package; the multi-process tests supply their own CPU stand-in
for the two local calls.

Every rank returns a consecutive slice of the suffix array; the slices in rank
order are the whole suffix array (`gather_sa`).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist


# ---------------------------------------------------------------------------
# local steps
# ---------------------------------------------------------------------------
class DeviceOps:
    """Local steps on the rank's GPU through the library's C ABI."""

    def __init__(self, ctx, device):
        self.ctx = ctx
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("DeviceOps works on CUDA tensors")

    def argsort_words(self, words):
        """Stable lexicographic argsort of rows given as uint32 values in int64
        tensors, words[-1] most significant: least significant groups of up to
        three words first, each a stable radix sort carrying the permutation."""
        n = words[0].numel()
        perm = torch.arange(n, dtype=torch.int32, device=self.device)
        if n <= 1:
            return perm.to(torch.int64)
        torch.cuda.synchronize(self.device)  # the library's stream does not wait for torch's
        for g in range(0, len(words), 3):
            chunk = words[g:g + 3]
            keys = [w.index_select(0, perm.to(torch.int64)).to(torch.int32).contiguous() for w in chunk]
            self.ctx.sort_u32_device([k.data_ptr() for k in keys], perm.data_ptr(), n)
        return perm.to(torch.int64)

    def suffix_array(self, s, sigma: int):
        """SA of a string of int64 symbols in [1, sigma]."""
        n = s.numel()
        if n == 0:
            return torch.zeros(0, dtype=torch.int64, device=self.device)
        t = s.to(torch.int32).contiguous()
        out = torch.empty(n, dtype=torch.int32, device=self.device)
        torch.cuda.synchronize(self.device)
        self.ctx.build_sa_u32_device(t.data_ptr(), n, int(sigma), out.data_ptr(), dc=3, sa_width=32)
        return out.to(torch.int64)


# ---------------------------------------------------------------------------
# exchange
# ---------------------------------------------------------------------------
class Comm:
    """The collectives the build needs, on one process group."""

    def __init__(self, group=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def allgather_i64(self, values, device):
        """Every rank's fixed-length int64 vector: tensor [world, len]."""
        t = torch.as_tensor(values, dtype=torch.int64, device=device).reshape(-1)
        out = [torch.empty_like(t) for _ in range(self.world)]
        dist.all_gather(out, t, group=self.group)
        return torch.stack(out)

    def allreduce_i64(self, value: int, device, op=dist.ReduceOp.SUM) -> int:
        t = torch.tensor([int(value)], dtype=torch.int64, device=device)
        dist.all_reduce(t, op=op, group=self.group)
        return int(t.item())

    def alltoallv(self, arrays, dest, device):
        """Sends element k of every array in `arrays` (1-D, same length) to rank
        dest[k] (non-decreasing is not required).  Returns the arrays received,
        ordered by source rank, each source's elements in their sent order."""
        order = torch.argsort(dest, stable=True)
        counts = torch.bincount(dest, minlength=self.world)
        send_counts = counts.to(torch.int64)
        recv_counts = torch.empty_like(send_counts)
        dist.all_to_all_single(recv_counts, send_counts, group=self.group)
        sc, rc = send_counts.tolist(), recv_counts.tolist()
        out = []
        for a in arrays:
            src = a.index_select(0, order).contiguous()
            r = torch.empty(sum(rc), dtype=a.dtype, device=device)
            dist.all_to_all_single(r, src, rc, sc, group=self.group)
            out.append(r)
        return out

    def gather_to_root(self, t, device):
        """Concatenation of every rank's 1-D int64 tensor on rank 0 (others: None)."""
        n = self.allgather_i64([t.numel()], device)[:, 0].tolist()
        big = max(n) if n else 0
        pad = torch.zeros(big, dtype=torch.int64, device=device)
        pad[: t.numel()] = t
        out = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(out, pad, group=self.group)
        if self.rank != 0:
            return None
        return torch.cat([o[:k] for o, k in zip(out, n)])


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
@dataclass
class _Dc:
    X: int
    D: int
    dc: list            # the difference cover, ascending
    in_dc: torch.Tensor  # [X] bool
    next_rank: list     # index of the first cover element >= c (D: the next block's first)
    cmp: torch.Tensor    # [X, X, 3] (d, r1, r2) of merge_samples.hpp's comparator


def _dc(X: int, device) -> _Dc:
    from . import dc_table
    dcs, nr, cmp = dc_table(X)
    in_dc = torch.zeros(X, dtype=torch.bool, device=device)
    in_dc[torch.as_tensor(dcs.astype(np.int64), device=device)] = True
    return _Dc(X, len(dcs), [int(v) for v in dcs], in_dc, [int(v) for v in nr],
               torch.as_tensor(cmp.astype(np.int64), device=device))


def _starts(n: int, world: int):
    """First position of each rank's block (the last rank also owns position n)."""
    return [r * n // world for r in range(world)]


def _owner(pos, starts_t):
    return torch.searchsorted(starts_t, pos, right=True) - 1


def _chars_per_word(B: int) -> int:
    c = 1
    while B ** (c + 1) <= (1 << 32):
        c += 1
    return c


def _window_words(ext, idx, L: int, B: int):
    """Windows ext[idx : idx + L] (base-B symbols, 0 past the end) as uint32
    words in int64 tensors, least significant word first."""
    cpw = _chars_per_word(B)
    W = (L + cpw - 1) // cpw
    words = []
    for k in range(W):
        acc = torch.zeros(idx.numel(), dtype=torch.int64, device=idx.device)
        for j in range(cpw):
            acc = acc * B
            if k * cpw + j < L:
                acc = acc + ext.index_select(0, idx + (k * cpw + j))
        words.append(acc)
    return words[::-1]


def _rows_greater(words, split):
    """words (least significant first) > split (list of ints, same order), lexicographically."""
    gt = torch.zeros(words[0].numel(), dtype=torch.bool, device=words[0].device)
    eq = torch.ones_like(gt)
    for w, s in zip(reversed(words), reversed(split)):
        gt = gt | (eq & (w > s))
        eq = eq & (w == s)
    return gt


def _rows_equal_prev(words):
    """Row k equals row k-1 (row 0: False)."""
    n = words[0].numel()
    eq = torch.zeros(n, dtype=torch.bool, device=words[0].device)
    if n > 1:
        e = torch.ones(n - 1, dtype=torch.bool, device=words[0].device)
        for w in words:
            e = e & (w[1:] == w[:-1])
        eq[1:] = e
    return eq


def _halo(comm: Comm, t_loc, H: int, device):
    """The H symbols after this rank's block (zeros past the text's end), from
    the first symbols of the following ranks' blocks."""
    head = torch.zeros(H, dtype=torch.int64, device=device)
    k = min(H, t_loc.numel())
    head[:k] = t_loc[:k]
    heads = comm.allgather_i64(head, device)
    lens = comm.allgather_i64([t_loc.numel()], device)[:, 0].tolist()
    parts, need = [], H
    for r in range(comm.rank + 1, comm.world):
        if need == 0:
            break
        take = min(lens[r], need)
        if take:
            parts.append(heads[r, :take])
            need -= take
    if need:
        parts.append(torch.zeros(need, dtype=torch.int64, device=device))
    return torch.cat(parts) if parts else torch.zeros(0, dtype=torch.int64, device=device)


def _sample_sort(comm: Comm, ops, words, pos, device):
    """Distributed sort of rows (words least significant first) carrying pos:
    local sort, p - 1 splitters from a regular sample of every rank, an
    alltoallv by bucket, local sort of what arrived (sample_sort.hpp:36-171).
    A row goes to the number of splitters it exceeds, so equal rows always
    meet on one rank.  Returns this rank's rows in global order."""
    perm = ops.argsort_words(words)
    words = [w.index_select(0, perm) for w in words]
    pos = pos.index_select(0, perm)
    p = comm.world
    if p == 1:
        return words, pos
    W = len(words)
    nloc = pos.numel()
    S = 32 * p
    take = min(nloc, S)
    samp = torch.zeros((S, W + 1), dtype=torch.int64, device=device)
    if take:
        si = (torch.arange(take, device=device) * nloc) // take
        samp[:take, 0] = 1
        for k, w in enumerate(words):
            samp[:take, 1 + k] = w.index_select(0, si)
    allv = comm.allgather_i64(samp.reshape(-1), device).reshape(p * S, W + 1)
    allv = allv[allv[:, 0] == 1]
    dest = torch.zeros(nloc, dtype=torch.int64, device=device)
    total = allv.shape[0]
    if total:
        cols = [allv[:, 1 + k].contiguous() for k in range(W)]
        order = ops.argsort_words(cols)
        srt = allv.index_select(0, order)
        for j in range(p - 1):
            row = srt[min(total - 1, ((j + 1) * total) // p), 1:].tolist()
            dest += _rows_greater(words, row).to(torch.int64)
    recv = comm.alltoallv(words + [pos], dest, device)
    words, pos = recv[:W], recv[W]
    perm = ops.argsort_words(words)
    return [w.index_select(0, perm) for w in words], pos.index_select(0, perm)


def _exchange_lookup(comm: Comm, req_pos, starts_t, table, lo: int, device):
    """table[q - lo] on the owner of every requested position q (all positions
    owned by some rank): one alltoallv of the requests, one of the answers."""
    me = torch.full_like(req_pos, comm.rank)
    tag = torch.arange(req_pos.numel(), dtype=torch.int64, device=device)
    q, src, t = comm.alltoallv([req_pos, me, tag], _owner(req_pos, starts_t), device)
    val = table.index_select(0, q - lo) if q.numel() else q
    back_tag, back_val = comm.alltoallv([t, val], src, device)
    out = torch.empty_like(req_pos)
    out[back_tag] = back_val
    return out


def _recurse(comm: Comm, ops, spos, names, n: int, dc: _Dc, sigma: int, base_threshold: int, device):
    """Ranks of the samples from the suffix array of their names in
    (i mod X, i div X) order (compute_ranks.hpp:49-56, pdcx.hpp:146-212,
    map_back pdcx.hpp:83-94).  Returns (sample positions, ranks), anywhere."""
    X, D = dc.X, dc.D
    num = [((n - r) // X + 1) if r <= n else 0 for r in dc.dc]
    sb = [0]
    for c in range(D):
        sb.append(sb[-1] + num[c])
    m = sb[D]
    inv = torch.full((X,), -1, dtype=torch.int64, device=device)
    inv[torch.tensor(dc.dc, dtype=torch.int64, device=device)] = torch.arange(D, dtype=torch.int64, device=device)
    sb_t = torch.tensor(sb, dtype=torch.int64, device=device)
    q = sb_t.index_select(0, inv.index_select(0, spos % X)) + spos // X
    startsR = _starts(m, comm.world)
    sR = torch.tensor(startsR, dtype=torch.int64, device=device)
    rq, rname = comm.alltoallv([q, names], _owner(q, sR), device)
    loR = startsR[comm.rank]
    hiR = startsR[comm.rank + 1] if comm.rank + 1 < comm.world else m
    r_loc = torch.zeros(hiR - loR, dtype=torch.int64, device=device)
    r_loc[rq - loR] = rname
    sa_r = _level(comm, ops, r_loc, m, sigma, X, base_threshold, device)
    lens = comm.allgather_i64([sa_r.numel()], device)[:, 0]
    off = int(lens[: comm.rank].sum().item())
    ranks = off + 1 + torch.arange(sa_r.numel(), dtype=torch.int64, device=device)
    c = torch.searchsorted(sb_t[1:], sa_r, right=True)
    dct = torch.tensor(dc.dc, dtype=torch.int64, device=device)
    return (sa_r - sb_t.index_select(0, c)) * X + dct.index_select(0, c), ranks


# rows of the tie break evaluated at once (pairs of one tie group's members)
_PAIR_CHUNK = 1 << 24


def _tie_break(pos, gid, rk, dc: _Dc, device):
    """Orders every tie group (equal windows) with the difference-cover
    comparator: i before j iff ranks_i[r1] < ranks_j[r2] for
    (d, r1, r2) = cmpDepthRanks[i mod X][j mod X] (merge_samples.hpp:87-109),
    where ranks_i are the ranks of the D samples at or after i.  Each member's
    place in its group is the number of members before it under the
    comparator, counted over the group's pairs in chunks."""
    T = pos.numel()
    if T == 0:
        return pos
    first = torch.ones(T, dtype=torch.bool, device=device)
    first[1:] = gid[1:] != gid[:-1]
    gstart = torch.cummax(torch.where(first, torch.arange(T, device=device), torch.zeros_like(gid)), 0).values
    gsize = torch.bincount(gid - gid[0])
    gsz = gsize.index_select(0, gid - gid[0])
    cls = pos % dc.X
    less = torch.zeros(T, dtype=torch.int64, device=device)
    csum = torch.cumsum(gsz, 0)
    e0 = 0
    while e0 < T:
        base = int(csum[e0 - 1].item()) if e0 else 0
        e1 = int(torch.searchsorted(csum, torch.tensor(base + _PAIR_CHUNK, device=device), right=True).item())
        e1 = max(e1, e0 + 1)
        e = torch.arange(e0, min(e1, T), device=device)
        reps = gsz.index_select(0, e)
        ee = torch.repeat_interleave(e, reps)
        within = torch.arange(ee.numel(), device=device) - torch.repeat_interleave(torch.cumsum(reps, 0) - reps, reps)
        ff = gstart.index_select(0, ee) + within
        tab = dc.cmp[cls.index_select(0, ff), cls.index_select(0, ee)]  # f before e?
        rf = rk[ff, tab[:, 1]]
        re = rk[ee, tab[:, 2]]
        less.index_add_(0, ee, (rf < re).to(torch.int64))
        e0 = int(e[-1].item()) + 1
    out = torch.empty_like(pos)
    out[gstart + less] = pos
    return out


def _level(comm: Comm, ops, t_loc, n: int, sigma: int, X: int, base_threshold: int, device):
    """This rank's slice of the SA of the block-distributed string T (t_loc =
    its block, symbols in [1, sigma]; rank r holds T[r*n//p, (r+1)*n//p))."""
    p, r = comm.world, comm.rank
    if n <= base_threshold:  # small strings: one local build on rank 0 (pdcx.hpp:115-124)
        full = comm.gather_to_root(t_loc, device)
        if r == 0:
            return ops.suffix_array(full, sigma)
        return torch.zeros(0, dtype=torch.int64, device=device)
    dc = _dc(X, device)
    D, L = dc.D, X
    starts = _starts(n, p)
    lo = starts[r]
    last = r == p - 1
    cnt = t_loc.numel() + (1 if last else 0)  # the last rank also holds the empty suffix n
    starts_t = torch.tensor(starts, dtype=torch.int64, device=device)
    # phase 1 + 4 window sort of every suffix (the last L - 1 read the halo)
    ext = torch.cat([t_loc, _halo(comm, t_loc, L + X, device), torch.zeros(L + X, dtype=torch.int64, device=device)])
    idx = torch.arange(cnt, dtype=torch.int64, device=device)
    words, pos = _sample_sort(comm, ops, _window_words(ext, idx, L, sigma + 1), lo + idx, device)
    head = ~_rows_equal_prev(words)
    if head.numel():
        head[0] = True  # equal windows never span two ranks
    gid = torch.cumsum(head.to(torch.int64), 0) - 1
    del words
    # phase 2: names of the samples (1 + distinct windows before), unique offsets over ranks
    is_s = dc.in_dc.index_select(0, pos % X)
    s_idx = torch.nonzero(is_s).flatten()
    sg = gid.index_select(0, s_idx)
    change = torch.ones(sg.numel(), dtype=torch.int64, device=device)
    if sg.numel() > 1:
        change[1:] = (sg[1:] != sg[:-1]).to(torch.int64)
    counts = comm.allgather_i64([sg.numel(), int(change.sum().item())], device)
    m = int(counts[:, 0].sum().item())
    distinct = int(counts[:, 1].sum().item())
    names = int(counts[:r, 1].sum().item()) + torch.cumsum(change, 0)
    spos = pos.index_select(0, s_idx)
    # phase 3: ranks of the samples, by name or by recursion
    if distinct < m:
        spos, names = _recurse(comm, ops, spos, names, n, dc, distinct, base_threshold, device)
    rp, rr = comm.alltoallv([spos, names], _owner(spos, starts_t), device)
    rank_loc = torch.zeros(cnt, dtype=torch.int64, device=device)
    rank_loc[rp - lo] = rr
    # phase 4: D ranks of the samples at or after every tied suffix, then the comparator
    gsize = torch.bincount(gid) if gid.numel() else gid
    tied = gsize.index_select(0, gid) >= 2 if gid.numel() else gid.bool()
    t_idx = torch.nonzero(tied).flatten()
    if comm.allreduce_i64(t_idx.numel(), device) > 0:
        tpos = pos.index_select(0, t_idx)
        nr = torch.tensor(dc.next_rank, dtype=torch.int64, device=device).index_select(0, tpos % X)
        dct = torch.tensor(dc.dc, dtype=torch.int64, device=device)
        j = nr[:, None] + torch.arange(D, device=device)[None, :]
        sp = ((tpos // X)[:, None] + j // D) * X + dct.index_select(0, (j % D).reshape(-1)).reshape(j.shape)
        flat = sp.reshape(-1)
        inside = flat <= n
        rk = torch.zeros_like(flat)
        rk[inside] = _exchange_lookup(comm, flat[inside], starts_t, rank_loc, lo, device)
        new = _tie_break(tpos, gid.index_select(0, t_idx), rk.reshape(-1, D), dc, device)
        pos = pos.clone()
        pos[t_idx] = new
    return pos[pos != n]


def _remap(comm: Comm, block, device):
    """Bytes present anywhere in the text mapped to 1..sigma (cli.cpp:417-463)."""
    h = torch.bincount(block.to(torch.int64), minlength=256)
    dist.all_reduce(h, group=comm.group)
    present = h > 0
    table = torch.cumsum(present.to(torch.int64), 0)
    return table.index_select(0, block.to(torch.int64)), int(present.sum().item())


def build_sa_distributed(block, n: int, dc: int = 39, ops=None, group=None, base_threshold: int = 1 << 22):
    """This rank's slice of the suffix array of a text of n bytes held in
    blocks: rank r passes T[r*n//p, (r+1)*n//p) as a uint8 tensor on its device
    (the reference's block distribution, mpi/io.hpp:33-65).  Collective over
    the process group.  Returns int64 positions; the slices in rank order form
    the suffix array.  ops: the local steps (default: DeviceOps on the block's
    GPU); strings of at most base_threshold symbols are built on rank 0."""
    comm = Comm(group)
    device = block.device
    starts = _starts(n, comm.world) + [n]
    want = starts[comm.rank + 1] - starts[comm.rank]
    if block.numel() != want:
        raise ValueError(f"rank {comm.rank} holds {block.numel()} bytes, its block has {want}")
    if ops is None:
        if device.type != "cuda":
            raise RuntimeError("the distributed build runs on GPUs: pass a CUDA block")
        from . import Context
        ops = DeviceOps(Context(device.index or 0), device)
    if base_threshold < 1:
        raise ValueError("base_threshold must be at least 1")
    t, sigma = _remap(comm, block, device)
    return _level(comm, ops, t, n, max(sigma, 1), dc, base_threshold, device)


def gather_sa(local, group=None):
    """The whole suffix array on rank 0 (None elsewhere)."""
    return Comm(group).gather_to_root(local, local.device)
