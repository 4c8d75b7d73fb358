"""Host-side checks of the persistent network launch's schedule (csrc/cnn_net.cu): the tile
numbering restated from the kernel's decode(), and the properties its waits rely on.

Tiles of layers base .. L-1 are numbered layer by layer (image, rotated tile row, strip); CTA c of
G takes tiles c, c + G, ... in order.  A tile of layer l > base waits for tile rows t-1, t, t+1
(periodic) of layer l-1 in every strip.  The checks: the numbering is a bijection; every input of
a tile has a smaller number (so the smallest unfinished tile can always run); the tiles that read
a row of the buffer a tile overwrites are among its own inputs (buffer reuse is ordered by the
same waits); and a discrete-event run of G round-robin CTAs, each with an in-order pipeline of
a few tiles in flight, finishes every tile for several shapes."""
import itertools
import random

import pytest


def decode(item, B, T, S, base):
    """Mirror of the kernel's decode(): (layer, image, tile row, strip) of a tile number."""
    per_layer = B * T * S
    j, r = divmod(item, per_layer)
    b, r = divmod(r, T * S)
    pos, xs = divmod(r, S)
    return j + base, b, (pos + j) % T, xs


def inputs(tile, T, S, base):
    """The (layer, image, row) counters a tile waits for, each needing every strip."""
    l, b, t, _ = tile
    if l <= base:
        return []
    return [(l - 1, b, (t + d) % T) for d in (-1, 0, 1)]


SHAPES = [(1, 192, 3, 6, 1), (2, 3, 1, 4, 1), (1, 2, 2, 5, 1), (3, 1, 1, 3, 1), (1, 4, 1, 8, 1), (2, 5, 2, 6, 0)]


@pytest.mark.parametrize("B,T,S,L,base", SHAPES)
def test_numbering_is_a_bijection_and_inputs_come_first(B, T, S, L, base):
    total = (L - base) * B * T * S
    tiles = [decode(i, B, T, S, base) for i in range(total)]
    assert len(set(tiles)) == total
    assert set(tiles) == set(itertools.product(range(base, L), range(B), range(T), range(S)))
    number = {tile: i for i, tile in enumerate(tiles)}
    for i, tile in enumerate(tiles):
        for (l, b, t) in inputs(tile, T, S, base):
            for xs in range(S):
                assert number[(l, b, t, xs)] < i


@pytest.mark.parametrize("B,T,S,L,base", SHAPES)
def test_buffer_reuse_is_covered_by_the_inputs(B, T, S, L, base):
    """Layer l writes the buffer layer l-2 wrote; layer l-1's tiles read rows t'-1 .. t'+2 of the
    padded halo, i.e. image rows of tile rows t'-1 .. t'+1.  Every layer l-1 tile that reads a
    row layer l's tile (l, b, t) overwrites must be one of that tile's inputs."""
    for l in range(base + 2, L):
        for b, t in itertools.product(range(B), range(T)):
            needed = set(inputs((l, b, t, 0), T, S, base))
            # layer l-1 tiles whose halo covers tile row t (their rows t'-1, t', t'+1)
            readers = {(l - 1, b, tp) for tp in range(T) if t in {(tp + d) % T for d in (-1, 0, 1)}}
            assert readers <= needed


@pytest.mark.parametrize("B,T,S,L,base,G,depth", [(1, 192, 3, 6, 1, 148, 4), (1, 192, 3, 6, 1, 37, 4),
                                                  (2, 3, 1, 4, 1, 6, 4), (1, 2, 2, 5, 1, 3, 2),
                                                  (1, 8, 3, 8, 1, 148, 4), (2, 5, 2, 6, 0, 7, 3)])
def test_round_robin_ctas_finish_every_tile(B, T, S, L, base, G, depth):
    """Discrete-event run: each CTA takes its tiles in order, keeps up to `depth` in flight (the
    halo stages), starts a tile only when its inputs are complete and completes tiles in order
    after a random latency.  Every tile completes (no wait can be left hanging)."""
    rng = random.Random(B * 1000 + T * 10 + G)
    total = (L - base) * B * T * S
    tiles = [decode(i, B, T, S, base) for i in range(total)]
    done_rows = {}
    queues = {c: list(range(c, total, G)) for c in range(G)}
    inflight = {c: [] for c in range(G)}  # (finish time, item)
    now, finished = 0, 0
    while finished < total:
        progressed = False
        for c in range(G):
            q, fl = queues[c], inflight[c]
            while q and len(fl) < depth:
                need = inputs(tiles[q[0]], T, S, base)
                if any(done_rows.get(key, 0) < S for key in need):
                    break
                start = max([now] + [f for f, _ in fl])  # the pipeline keeps tiles in order
                fl.append((start + rng.randint(1, 5), q.pop(0)))
                progressed = True
            while fl and fl[0][0] <= now:
                _, item = fl.pop(0)
                l, b, t, _ = tiles[item]
                done_rows[(l, b, t)] = done_rows.get((l, b, t), 0) + 1
                finished += 1
                progressed = True
        if not progressed and not any(inflight.values()):
            pytest.fail(f"stuck with {total - finished} tiles left")
        now += 1
    assert all(v == S for v in done_rows.values())
