"""The fused proposal net's mbarrier protocol (lp_net_kernel in
csrc/learned.cu), restated as a schedule and run under random
interleavings on the CPU: no agent deadlocks, and every parity wait
(mbarrier.try_wait.parity) sees its barrier either one phase short of the
awaited one or past it, never further behind (the wait would then hang) or
two phases short (the parity would alias and the wait pass early).

The agents: ISSUERS MMA-issuing warps taking the tiles t = i, i + ISSUERS,
... of the 4 x 9 tiles of each map; one epilogue group consuming every
tile in order. Barriers: full/empty per accumulator slot (seq % NSLOT,
seq = 36 j + t), a stored barrier per (layer, tile), the input-ready and
bulk-copy barriers. The constants are read from the kernel source."""
import os
import random
import re

import pytest

SRC = os.path.join(os.path.dirname(__file__), "..", "oxideav-vp8_b200", "csrc", "learned.cu")


def kernel_constants():
    text = open(SRC).read()
    ns = text[text.index("namespace lpnet {"):text.index("}  // namespace lpnet")]

    def const(name):
        return int(re.search(rf"constexpr int {name} = (\d+);", ns).group(1))

    return const("TILES"), const("NSLOT"), const("ISSUERS")


TILES, NSLOT, ISSUERS = kernel_constants()
PER_MAP = 4 * TILES


def slot(j, t):
    seq = PER_MAP * j + t
    return seq % NSLOT, seq // NSLOT


def issuer(i, maps, stored, issuers):
    if i == 0:
        yield ("arrive", "stage")  # the first map's bulk copy
    for j in range(maps):
        yield ("wait", "input", j)
        if i == 0 and j + 1 < maps:
            yield ("arrive", "stage")
        for t in range(i, PER_MAP, issuers):
            layer, u = divmod(t, TILES)
            if layer > 0:
                for w in (u - 1, u, u + 1):
                    if 0 <= w < TILES:
                        b, c = stored(j, layer - 1, w)
                        yield ("wait", b, c)
            s, use = slot(j, t)
            if use > 0:
                yield ("wait", f"empty{s}", use - 1)
            yield ("arrive", f"full{s}")


def epilogue(maps, stored):
    yield ("wait", "stage", 0)
    yield ("arrive", "input")
    for j in range(maps):
        for t in range(3 * TILES):
            s, use = slot(j, t)
            yield ("wait", f"full{s}", use)
            yield ("arrive", f"empty{s}")
            yield ("arrive", stored(j, t // TILES, t % TILES)[0])
        for u in range(TILES):
            s, use = slot(j, 3 * TILES + u)
            yield ("wait", f"full{s}", use)
            yield ("arrive", f"empty{s}")
            if u == 0 and j + 1 < maps:
                yield ("wait", "stage", j + 1)
                yield ("arrive", "input")


def per_layer_tile(j, layer, u):
    """The kernel's scheme: one barrier per (layer, tile), once a map."""
    return f"stored{layer}_{u}", j


def shared_across_layers(j, layer, u):
    """One barrier per tile reused by the three layers (3 phases a map)."""
    return f"stored{u}", 3 * j + layer


def run(maps, seed, stored, issuers=ISSUERS):
    rnd = random.Random(seed)
    done_phases = {}
    agents = [issuer(i, maps, stored, issuers) for i in range(issuers)] + [epilogue(maps, stored)]
    cur = [next(a) for a in agents]
    live = [True] * len(agents)
    while any(live):
        ready = []
        for i, op in enumerate(cur):
            if not live[i]:
                continue
            if op[0] == "arrive":
                ready.append(i)
                continue
            _, b, c = op
            n = done_phases.get(b, 0)
            if n > c + 1:
                raise AssertionError(f"missed phase: agent {i} waits phase {c} of {b}, {n} done")
            if ((n & 1) != (c & 1)) != (n >= c + 1):
                raise AssertionError(f"parity alias: agent {i} waits phase {c} of {b}, {n} done")
            if n >= c + 1:
                ready.append(i)
        if not ready:
            raise AssertionError(f"deadlock: {cur}")
        i = rnd.choice(ready)
        if cur[i][0] == "arrive":
            done_phases[cur[i][1]] = done_phases.get(cur[i][1], 0) + 1
        try:
            cur[i] = next(agents[i])
        except StopIteration:
            live[i] = False


def test_constants_fit_the_protocol():
    # A slot's tiles come from one issuer: NSLOT a multiple of ISSUERS.
    assert NSLOT % ISSUERS == 0 and PER_MAP == 36


@pytest.mark.parametrize("maps", [1, 2, 3, 5])
def test_protocol_has_no_deadlock_and_no_parity_alias(maps):
    for seed in range(150):
        run(maps, seed, per_layer_tile)


@pytest.mark.parametrize("issuers", [1, 2, 4, 8])
def test_protocol_holds_for_other_issuer_counts(issuers):
    for seed in range(60):
        run(3, seed, per_layer_tile, issuers)


def test_the_check_catches_a_barrier_shared_across_layers():
    # With two issuers, a stored barrier reused by the three layers can
    # complete twice before the lagging issuer waits on it (the other
    # issuer's tiles let the epilogue finish the next layer's tile first).
    with pytest.raises(AssertionError, match="missed phase|parity alias|deadlock"):
        for seed in range(2000):
            run(3, seed, shared_across_layers, issuers=2)
