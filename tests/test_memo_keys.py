"""The exactness argument of the cycle memo, checked on the CPU with a Python restatement of the key
functions in csrc/war_refill.cuh (memo_key_state, memo_slot, path_entry) and csrc/war_held.cu (h_key):
different positions get different keys, a position and its mirror image share one, and a path entry
together with its slot gives back exactly the key that wrote it (multiplication by an odd constant is a
bijection of 64-bit words)."""
import random

M64 = (1 << 64) - 1
MUL = 0x9E3779B97F4A7C15


def sentinel(cards):
    w = 0
    for i, c in enumerate(cards):
        w |= c << (4 * i)
    return w | (1 << (4 * len(cards)))


def pile_len(w):
    return (w.bit_length() - 1) >> 2


def memo_key_state(w1, w2, n):
    h, o = (w2, w1) if w2 < w1 else (w1, w2)
    lh = pile_len(h)
    cat = ((h ^ (1 << (4 * lh))) | (o << (4 * lh))) & M64
    kb = 4 * (n - 1)
    return (cat & ((1 << kb) - 1)) | (lh << kb)


def memo_slot(key, bits):
    return ((key * MUL) & M64) >> (64 - bits)


def path_entry(key, bits, v):
    return ((((key * MUL) & M64) << bits) & M64) | v


def key_back(slot, entry, bits):
    h = ((slot << (64 - bits)) | (entry >> bits)) & M64
    return (h * pow(MUL, -1, 1 << 64)) & M64


def h_key(wh, wo, lh, p, n):
    cat = (wh | (wo << (4 * lh))) & M64
    if n < 17:
        kb = 4 * (n - 2)
        return (cat & ((1 << kb) - 1)) | (lh << kb) | (p << (kb + 4))
    c0, c1, c2 = (cat >> 52) & 15, (cat >> 56) & 15, (cat >> 60) & 15
    order = 2 * (int(c0 > c1) + int(c0 > c2)) + int(c1 > c2)
    return (cat & ((1 << 52) - 1)) | (order << 52) | (lh << 55) | (p << 59)


def random_position(rnd, n):
    cards = list(range(n))
    rnd.shuffle(cards)
    k = rnd.randint(1, n - 1)
    return cards[:k], cards[k:]


def test_state_keys_are_injective_and_mirror_symmetric():
    rnd = random.Random(1)
    for n in (5, 9, 13, 15, 16):
        seen = {}
        for _ in range(20000):
            a, b = random_position(rnd, n)
            w1, w2 = sentinel(a), sentinel(b)
            k = memo_key_state(w1, w2, n)
            assert k < (1 << 64) and k != 0
            assert k == memo_key_state(w2, w1, n)                   # the same game with the players swapped
            pos = frozenset([tuple(a), tuple(b)])
            assert seen.setdefault(k, pos) == pos, (n, a, b)        # one key, one position (up to the swap)


def test_path_entry_names_its_key():
    rnd = random.Random(2)
    for bits in (12, 20, 30, 31):
        for _ in range(2000):
            key = rnd.getrandbits(64)
            v = rnd.randrange(1, 1 << bits)
            e = path_entry(key, bits, v)
            assert e & ((1 << bits) - 1) == v and e != 0
            assert key_back(memo_slot(key, bits), e, bits) == key
            # another key in the same slot can not match this entry
            other = rnd.getrandbits(64)
            if other != key and memo_slot(other, bits) == memo_slot(key, bits):
                assert (e ^ path_entry(other, bits, 0)) >> bits != 0


def test_held_keys_are_injective():
    rnd = random.Random(3)
    for n in (9, 16, 17):
        seen = {}
        for _ in range(20000):
            others = list(range(n - 1))
            rnd.shuffle(others)
            lh = rnd.randint(0, n - 2)
            p = rnd.randint(0, lh)
            wh = sum(c << (4 * i) for i, c in enumerate(others[:lh]))
            wo = sum(c << (4 * i) for i, c in enumerate(others[lh:]))
            k = h_key(wh, wo, lh, p, n)
            assert k < (1 << 64)
            pos = (tuple(others[:lh]), tuple(others[lh:]), p)
            assert seen.setdefault(k, pos) == pos, (n, pos)
