"""Seeded synthetic LTL-learning instances.

The reference ships no generator, so its benchmark shapes are reproduced here
from seeds: a random hidden formula labels Bernoulli traces, and traces are
accepted in draw order until the positive and negative quotas are met.

Operator semantics used to label traces are the reference's characteristic-set
(CS) bit tricks (code/ltli6463.cu:203-204, :295, :385, :468, :551-556,
:638-645, :739-752); bit k of a trace's word is position k, and a trace is
labelled positive when the hidden formula holds at position 0.

Every instance is a plain record of arrays:
  steps    uint32[total_steps]  bit (letter - 'a') set when the letter holds
  offsets  int32[n + 1]         trace t owns steps[offsets[t]:offsets[t+1]]
  num_pos, num_neg              positives first, then negatives
  alphabet str                  the letters, sorted (the reference's std::set)
"""
from __future__ import annotations

import dataclasses
import numpy as np

UNARY = ("~", "X", "F", "G")
BINARY = ("&", "|", "U")
DEFAULT_LETTERS = "pqrstuvwxyzabcdefghijklmno"

_U64 = np.uint64
_ONE = _U64(1)


@dataclasses.dataclass
class Instance:
    num_pos: int
    num_neg: int
    alphabet: str
    steps: np.ndarray
    offsets: np.ndarray
    hidden: str = ""

    @property
    def n(self) -> int:
        return self.num_pos + self.num_neg

    @property
    def lengths(self) -> np.ndarray:
        return np.diff(self.offsets).astype(np.int32)

    def atom_cs(self) -> np.ndarray:
        """uint64[alphabet_size, n]: bit k of [j, t] = letter j holds at step k of trace t."""
        lens = self.lengths
        out = np.zeros((len(self.alphabet), self.n), dtype=np.uint64)
        idx = np.repeat(np.arange(self.n), lens)
        pos = (np.arange(len(self.steps)) - np.repeat(self.offsets[:-1], lens)).astype(np.uint64)
        for j, ch in enumerate(self.alphabet):
            bit = ((self.steps >> (ord(ch) - 97)) & 1).astype(np.uint64)
            np.bitwise_or.at(out[j], idx, bit << pos)
        return out

    def trace_lines(self) -> list[str]:
        """Scarlet lines ("1,0;0,1;...") in alphabet order, positives then negatives.  Each
        distinct step mask is formatted once."""
        steps = np.asarray(self.steps, dtype=np.uint32)
        bits = [1 << (ord(c) - 97) for c in self.alphabet]
        masks, inv = np.unique(steps, return_inverse=True)
        text = np.array([",".join("1" if int(m) & b else "0" for b in bits) for m in masks] or [""], dtype=object)
        tokens = text[inv.ravel()].tolist()
        offs = np.asarray(self.offsets).tolist()
        return [";".join(tokens[offs[t]:offs[t + 1]]) for t in range(self.n)]

    def to_scarlet(self) -> str:
        """Same layout as the reference driver writes (code/dc.py:8-21)."""
        lines = self.trace_lines()
        out = lines[:self.num_pos] + ["---"] + lines[self.num_pos:] + ["---", "All operators", "---",
                                                                        ",".join(self.alphabet)]
        return "\n".join(out)


# ---------------------------------------------------------------- formulas

def random_formula(rng: np.random.Generator, size: int, nprops: int):
    """Uniform choice of operator at each node; binary splits uniform over sizes."""
    if size <= 1:
        return ("p", int(rng.integers(nprops)))
    if size == 2:
        return (UNARY[int(rng.integers(4))], random_formula(rng, 1, nprops))
    k = int(rng.integers(7))
    if k < 4:
        return (UNARY[k], random_formula(rng, size - 1, nprops))
    a = int(rng.integers(1, size - 1))
    return (BINARY[k - 4], random_formula(rng, a, nprops), random_formula(rng, size - 1 - a, nprops))


def formula_str(f, letters: str) -> str:
    """Fully parenthesised form the reference prints (code/ltli6463.cu:877-928)."""
    op = f[0]
    if op == "p":
        return letters[f[1]]
    if op in UNARY:
        return f"{op}({formula_str(f[1], letters)})"
    return f"({formula_str(f[1], letters)}){op}({formula_str(f[2], letters)})"


def _smear(w):
    for k in (1, 2, 4, 8, 16, 32):
        w = w | (w >> _U64(k))
    return w


def _until(x, y):
    for k in (1, 2, 4, 8, 16):
        y = y | (x & (y >> _U64(k)))
        x = x & (x >> _U64(k))
    return y | (x & (y >> _U64(32)))


def eval_cs(f, atoms: np.ndarray, mask: np.ndarray) -> np.ndarray:
    """Characteristic set of f on every trace (uint64 per trace)."""
    op = f[0]
    if op == "p":
        return atoms[f[1]]
    if op == "~":
        return ~eval_cs(f[1], atoms, mask) & mask
    if op == "X":
        return eval_cs(f[1], atoms, mask) >> _ONE
    if op == "F":
        return _smear(eval_cs(f[1], atoms, mask))
    if op == "G":
        w = eval_cs(f[1], atoms, mask)
        return w & ~_smear(~w & mask)
    a = eval_cs(f[1], atoms, mask)
    b = eval_cs(f[2], atoms, mask)
    if op == "&":
        return a & b
    if op == "|":
        return a | b
    return _until(a, b)


# ---------------------------------------------------------------- traces

def _draw(rng, m, nprops, lmin, lmax, p_bit):
    lens = rng.integers(lmin, lmax + 1, size=m)
    bits = rng.random((m, lmax, nprops)) < p_bit
    live = np.arange(lmax)[None, :] < lens[:, None]
    bits &= live[:, :, None]
    weights = (_ONE << np.arange(lmax, dtype=np.uint64))
    atoms = np.stack([(bits[:, :, j].astype(np.uint64) * weights).sum(axis=1, dtype=np.uint64)
                      for j in range(nprops)])
    mask = (_ONE << lens.astype(np.uint64)) - _ONE
    return lens, bits, atoms, mask


def _pack(letters, lens_list, bits_list):
    lens = np.asarray(lens_list, dtype=np.int64)
    offsets = np.zeros(len(lens) + 1, dtype=np.int32)
    offsets[1:] = np.cumsum(lens)
    shifts = np.array([ord(c) - 97 for c in letters], dtype=np.uint32)
    steps = np.zeros(int(offsets[-1]), dtype=np.uint32)
    for t, (ln, b) in enumerate(zip(lens_list, bits_list)):
        steps[offsets[t]:offsets[t + 1]] = (b[:ln].astype(np.uint32) << shifts[None, :]).sum(axis=1, dtype=np.uint32)
    return steps, offsets


def generate(seed: int, nprops: int, npos: int, nneg: int, lmin: int, lmax: int,
             p_bit: float = 0.5, fsize: int = 5, batch: int = 4096,
             max_batches: int = 64, max_formulas: int = 200) -> Instance:
    """Hidden-formula instance: traces drawn in order, labelled at position 0."""
    assert 1 <= lmin <= lmax <= 63 and 1 <= nprops <= 26
    rng = np.random.default_rng(seed)
    letters = "".join(sorted(DEFAULT_LETTERS[:nprops]))
    for _ in range(max_formulas):
        f = random_formula(rng, fsize, nprops)
        pos_l, pos_b, neg_l, neg_b = [], [], [], []
        for _b in range(max_batches):
            lens, bits, atoms, mask = _draw(rng, batch, nprops, lmin, lmax, p_bit)
            lab = (eval_cs(f, atoms, mask) & _ONE).astype(bool)
            for i in range(batch):
                if lab[i]:
                    if len(pos_l) < npos:
                        pos_l.append(int(lens[i])); pos_b.append(bits[i])
                elif len(neg_l) < nneg:
                    neg_l.append(int(lens[i])); neg_b.append(bits[i])
                if len(pos_l) == npos and len(neg_l) == nneg:
                    break
            if len(pos_l) == npos and len(neg_l) == nneg:
                steps, offsets = _pack(letters, pos_l + neg_l, pos_b + neg_b)
                return Instance(npos, nneg, letters, steps, offsets, formula_str(f, letters))
    raise RuntimeError("could not fill the positive/negative quotas")


def generate_hamming(seed: int, nprops: int, npos: int, nneg: int, lmin: int, lmax: int,
                     p_bit: float = 0.5, fsize: int = 6, flips=(1, 3), batch: int | None = None,
                     max_formulas: int = 200) -> Instance:
    """Near-miss instance: each negative is a positive with 1-3 bits flipped.

    Positives satisfy a hidden formula; a flipped copy becomes a negative only
    when the flip makes the hidden formula false and the copy is not equal to
    any positive, so a separating formula of bounded size always exists.
    """
    rng = np.random.default_rng(seed)
    letters = "".join(sorted(DEFAULT_LETTERS[:nprops]))
    if batch is None:  # traces drawn per round: enough for the quotas without oversized draws
        batch = min(4096, max(512, 8 * max(npos, nneg)))
    for _ in range(max_formulas):
        f = random_formula(rng, fsize, nprops)
        pos_l, pos_b = [], []
        for _b in range(64):
            lens, bits, atoms, mask = _draw(rng, batch, nprops, lmin, lmax, p_bit)
            lab = (eval_cs(f, atoms, mask) & _ONE).astype(bool)
            for i in np.nonzero(lab)[0][: npos - len(pos_l)]:
                pos_l.append(int(lens[i])); pos_b.append(bits[i])
            if len(pos_l) == npos:
                break
        if len(pos_l) < npos:
            continue
        seen = {(ln, b[:ln].tobytes()) for ln, b in zip(pos_l, pos_b)}
        neg_l, neg_b = [], []
        plen = np.asarray(pos_l, dtype=np.int64)
        pbits = np.stack(pos_b)
        weights = (_ONE << np.arange(lmax, dtype=np.uint64))
        for _round in range(200):
            if len(neg_l) >= nneg:
                break
            # a batch of flipped copies, evaluated together; kept in draw order
            src = rng.integers(npos, size=batch)
            lens = plen[src]
            bits = pbits[src].copy()
            nfl = rng.integers(flips[0], flips[1] + 1, size=batch)
            rows = np.arange(batch)
            for k in range(flips[1]):
                at = (rng.random(batch) * lens).astype(np.int64)
                prop = rng.integers(nprops, size=batch)
                act = nfl > k
                bits[rows[act], at[act], prop[act]] ^= True
            atoms = np.stack([(bits[:, :, j].astype(np.uint64) * weights).sum(axis=1, dtype=np.uint64)
                              for j in range(nprops)])
            mask = (_ONE << lens.astype(np.uint64)) - _ONE
            false_ = (eval_cs(f, atoms, mask) & _ONE) == 0
            for i in np.nonzero(false_)[0]:
                ln = int(lens[i])
                key = (ln, bits[i, :ln].tobytes())
                if key in seen:
                    continue
                seen.add(key)
                neg_l.append(ln); neg_b.append(bits[i])
                if len(neg_l) == nneg:
                    break
        if len(neg_l) == nneg:
            steps, offsets = _pack(letters, pos_l + neg_l, pos_b + neg_b)
            return Instance(npos, len(neg_l), letters, steps, offsets, formula_str(f, letters))
    raise RuntimeError("could not build a near-miss instance")


def generate_near_miss(seed: int, nprops: int, npos: int, nneg: int, lmin: int, lmax: int,
                       p_bit: float = 0.5, flips=(1, 3)) -> Instance:
    """Near-miss instance without a hidden formula: npos random positives (Bernoulli(p_bit)
    bits, lengths uniform lmin-lmax); each negative is a random positive with 1-3 random bits
    flipped, and a flipped copy equal to a positive (or to an earlier negative) is drawn
    again.  No separating formula of bounded size is planted."""
    rng = np.random.default_rng(seed)
    letters = "".join(sorted(DEFAULT_LETTERS[:nprops]))
    lens, bits, _, _ = _draw(rng, npos, nprops, lmin, lmax, p_bit)
    pos_l = [int(x) for x in lens]
    pos_b = [bits[i] for i in range(npos)]
    seen = {(ln, b[:ln].tobytes()) for ln, b in zip(pos_l, pos_b)}
    neg_l, neg_b = [], []
    for _ in range(1000 * max(1, nneg)):
        if len(neg_l) == nneg:
            break
        src = int(rng.integers(npos))
        ln = pos_l[src]
        b = pos_b[src].copy()
        for _k in range(int(rng.integers(flips[0], flips[1] + 1))):
            b[int(rng.integers(ln)), int(rng.integers(nprops))] ^= True
        key = (ln, b[:ln].tobytes())
        if key in seen:
            continue
        seen.add(key)
        neg_l.append(ln)
        neg_b.append(b)
    steps, offsets = _pack(letters, pos_l + neg_l, pos_b + neg_b)
    return Instance(npos, len(neg_l), letters, steps, offsets, "")


def hamming_neighbourhood(seed: int, nprops: int, length: int, delta: int = 1) -> Instance:
    """One random positive and every trace at Hamming distance exactly delta as negatives."""
    import itertools
    rng = np.random.default_rng(seed)
    letters = "".join(sorted(DEFAULT_LETTERS[:nprops]))
    b = rng.random((length, nprops)) < 0.5
    neg_b = []
    for cells in itertools.combinations(range(length * nprops), delta):
        c = b.copy()
        for cell in cells:
            c[cell // nprops, cell % nprops] ^= True
        neg_b.append(c)
    steps, offsets = _pack(letters, [length] * (1 + len(neg_b)), [b] + neg_b)
    return Instance(1, len(neg_b), letters, steps, offsets, "")


def from_scarlet_text(text: str) -> Instance:
    """Parse with the reference reader's rules (code/ltli6463.cu:1500-1573).

    The last line gives the letters (only a-z kept, file order maps values to
    letters); positives run until the first "---", negatives until the next.
    Inside a trace ';' ends a step, ',' is skipped, and every other character
    advances the value index, '1' marking the letter at that index.
    """
    lines = text.split("\n")
    if lines and lines[-1] == "":
        lines.pop()  # getline yields no line after a final newline
    body = text[:-1] if text.endswith("\n") else text
    k = body.rfind("\n")
    last = body[k + 1:] if k >= 0 else body
    alpha = [c for c in last if "a" <= c <= "z"]
    letters = "".join(sorted(set(alpha)))

    def parse_line(line):
        steps, cur, j = [], 0, 0
        for c in line:
            if c == ";":
                steps.append(cur); cur = 0; j = 0
            elif c == ",":
                continue
            else:
                if c == "1" and j < len(alpha):
                    cur |= 1 << (ord(alpha[j]) - 97)
                j += 1
        steps.append(cur)
        return steps

    it = iter(lines)
    pos, neg = [], []
    for line in it:
        if line == "---":
            break
        pos.append(parse_line(line))
    for line in it:
        if line == "---":
            break
        neg.append(parse_line(line))
    traces = pos + neg
    offsets = np.zeros(len(traces) + 1, dtype=np.int32)
    offsets[1:] = np.cumsum([len(t) for t in traces])
    steps = np.array([s for t in traces for s in t], dtype=np.uint32)
    return Instance(len(pos), len(neg), letters, steps, offsets)
