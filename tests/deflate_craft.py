"""Crafted DEFLATE streams for the inflate tests: an RFC 1951 encoder that
writes blocks of every type (stored, fixed, dynamic) with chosen code lengths,
so that codes of 1 to 15 bits, every length and distance symbol and empty
stored blocks occur.  zlib validates every crafted stream (tests/test_craft.py);
the GPU decoder must reproduce the bytes (tests/test_gpu_inflate.py)."""
import random

LEN_BASE = [3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258]
LEN_EXTRA = [0] * 8 + [1] * 4 + [2] * 4 + [3] * 4 + [4] * 4 + [5] * 4 + [0]
DIST_BASE = [1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129, 193, 257, 385, 513, 769, 1025, 1537, 2049, 3073,
             4097, 6145, 8193, 12289, 16385, 24577]
DIST_EXTRA = [0, 0, 0, 0] + [i // 2 for i in range(2, 28)]
CL_ORDER = [16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15]


class BitWriter:
    def __init__(self):
        self.out = bytearray()
        self.acc = 0
        self.n = 0

    def put(self, v, n):  # n bits of v, least significant first
        self.acc |= (v & ((1 << n) - 1)) << self.n
        self.n += n
        while self.n >= 8:
            self.out.append(self.acc & 0xFF)
            self.acc >>= 8
            self.n -= 8

    def code(self, c, n):  # a Huffman code: most significant bit first
        self.put(int(format(c, f"0{n}b")[::-1], 2), n)

    def align(self):
        if self.n:
            self.put(0, 8 - self.n)

    def bytes(self):
        self.align()
        return bytes(self.out)


def canonical(lengths):
    """Codes of RFC 1951 3.2.2 for the given lengths (0 = unused)."""
    bl = [0] * 16
    for l in lengths:
        bl[l] += 1
    bl[0] = 0
    nxt, code = [0] * 16, 0
    for b in range(1, 16):
        code = (code + bl[b - 1]) << 1
        nxt[b] = code
    codes = [0] * len(lengths)
    for s, l in enumerate(lengths):
        if l:
            codes[s] = nxt[l]
            nxt[l] += 1
    return codes


def tree_lengths(nsym, rng, short=None):
    """A complete set of code lengths (Kraft sum 1) with depths 1..15: leaves
    of a random binary tree grown by splitting leaves, deep ones preferred so
    that codes longer than 9 bits occur.  `short` gets the 1-bit code."""
    leaves = [1, 1]
    if short is not None:
        fixed, leaves = [1], [1]  # one child of the root stays a leaf
    else:
        fixed = []
    while len(leaves) + len(fixed) < nsym:
        cand = [i for i, d in enumerate(leaves) if d < 15]
        i = max(cand, key=lambda k: leaves[k]) if rng.random() < 0.3 else rng.choice(cand)
        d = leaves.pop(i)
        leaves += [d + 1, d + 1]
    depths = sorted(leaves)
    rng.shuffle(depths)
    if short is not None:
        depths.insert(short, 1)
    return depths


def dynamic_block(bw, tokens, lit_len, dist_len, final, used=None):
    bw.put(final, 1)
    bw.put(2, 2)
    bw.put(len(lit_len) - 257, 5)
    bw.put(len(dist_len) - 1, 5)
    bw.put(19 - 4, 4)
    cl_len = [4] * 16 + [0, 0, 0]  # symbols 0-15 with 4-bit codes, no repeats
    for s in CL_ORDER:
        bw.put(cl_len[s], 3)
    cl_code = canonical(cl_len)
    for l in list(lit_len) + list(dist_len):
        bw.code(cl_code[l], 4)
    emit_tokens(bw, tokens, canonical(lit_len), lit_len, canonical(dist_len), dist_len, used)


def fixed_block(bw, tokens, final):
    lit_len = [8] * 144 + [9] * 112 + [7] * 24 + [8] * 8
    dist_len = [5] * 30
    bw.put(final, 1)
    bw.put(1, 2)
    emit_tokens(bw, tokens, canonical(lit_len), lit_len, canonical(dist_len), dist_len)


def stored_block(bw, data, final):
    bw.put(final, 1)
    bw.put(0, 2)
    bw.align()
    bw.put(len(data), 16)
    bw.put(len(data) ^ 0xFFFF, 16)
    for b in data:
        bw.put(b, 8)


def emit_tokens(bw, tokens, lc, ll, dc, dl, used=None):
    """Writes the tokens and the end of block; `used` (a dict) collects the
    code lengths that occur: 'lit' and 'dist' sets."""
    for t in tokens:
        if isinstance(t, int):
            bw.code(lc[t], ll[t])
            if used is not None:
                used.setdefault("lit", set()).add(ll[t])
            continue
        length, dist = t
        i = max(k for k in range(29) if LEN_BASE[k] <= length)
        bw.code(lc[257 + i], ll[257 + i])
        bw.put(length - LEN_BASE[i], LEN_EXTRA[i])
        j = max(k for k in range(30) if DIST_BASE[k] <= dist)
        bw.code(dc[j], dl[j])
        if used is not None:
            used.setdefault("lit", set()).add(ll[257 + i])
            used.setdefault("dist", set()).add(dl[j])
        bw.put(dist - DIST_BASE[j], DIST_EXTRA[j])
    bw.code(lc[256], ll[256])


def random_tokens(rng, out, n, lit_weights=None, match_rate=0.3):
    """n tokens applied to `out` (bytearray); literals drawn with weights,
    matches with every length and distance the history allows."""
    toks = []
    lits = list(range(256))
    for _ in range(n):
        if len(out) >= 3 and rng.random() < match_rate:
            dist = rng.choice([rng.randint(1, min(len(out), 32768)), rng.randint(1, min(len(out), 40))])
            length = rng.choice([rng.randint(3, 258), rng.randint(3, 12)])
            for k in range(length):
                out.append(out[-dist])
            toks.append((length, dist))
        else:
            b = rng.choices(lits, lit_weights)[0] if lit_weights else rng.randrange(256)
            out.append(b)
            toks.append(b)
    return toks


def crafted_stream(seed, tokens=6000, used=None):
    """Blocks of every type with codes of 1 to 15 bits; returns (raw, data).
    `used` (a dict) collects the code lengths of the dynamic blocks."""
    rng = random.Random(seed)
    bw, out = BitWriter(), bytearray()
    plan = ["dyn", "fixed", "stored", "dyn1", "dyn", "stored0", "dyn1", "fixed"]
    for k, kind in enumerate(plan):
        final = int(k == len(plan) - 1)
        if kind.startswith("stored"):
            data = bytes(rng.randrange(256) for _ in range(0 if kind == "stored0" else rng.randint(1, tokens // 2)))
            out += data
            stored_block(bw, data, final)
        elif kind == "fixed":
            fixed_block(bw, random_tokens(rng, out, tokens // 2), final)
        else:
            one = kind == "dyn1"
            lit_len = tree_lengths(286, rng, short=rng.randrange(256) if one else None)
            dist_len = tree_lengths(30, rng)
            short = lit_len.index(1) if one else None
            weights = [50000 if b == short else 1 for b in range(256)] if one else None
            dynamic_block(bw, random_tokens(rng, out, tokens, weights, 0.05 if one else 0.3), lit_len, dist_len, final,
                          used)
    return bw.bytes(), bytes(out)


