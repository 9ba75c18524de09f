"""Constraint systems over 64-bit words: the reference's data model and wire format, plus a
generator of synthetic circuits with satisfying witnesses.

Mirrors verifier/core/src/constraint_system.rs: ShiftVariant (:50-100), ShiftedValueIndex
(:134-300), AndConstraint / MulConstraint, ValueVecLayout (:651-770), the v2 serialization
(:606-650; usize fields are u32 LE, words u64 LE) and validate_and_prepare's padding of the AND and
MUL constraint lists to powers of two (at least 8 and 1, :558-584).  The synthetic generator builds
layered chains of band / bxor / shifted-value operands and imul (the shapes the frontend's
CircuitBuilder emits: verifier/frontend/src/compiler/mod.rs) over seeded random words; every
constraint is satisfied by construction.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

SLL, SLR, SAR, ROTR, SLL32, SRL32, SRA32, ROTR32 = range(8)
MIN_AND_CONSTRAINTS = 8
MIN_MUL_CONSTRAINTS = 1

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


@dataclass(frozen=True)
class ShiftedValueIndex:
    value_index: int
    shift_variant: int = SLL
    amount: int = 0


@dataclass
class AndConstraint:
    a: list = field(default_factory=list)
    b: list = field(default_factory=list)
    c: list = field(default_factory=list)


@dataclass
class MulConstraint:
    a: list = field(default_factory=list)
    b: list = field(default_factory=list)
    hi: list = field(default_factory=list)
    lo: list = field(default_factory=list)


@dataclass
class ValueVecLayout:
    n_const: int
    n_inout: int
    n_witness: int
    n_internal: int
    offset_inout: int
    offset_witness: int
    committed_total_len: int
    n_scratch: int = 0


@dataclass
class OperandCSR:
    """Operands of a constraint list in CSR form: group g = constraint * k + operand slot
    (k = 3 for AND: a, b, c; k = 4 for MUL: a, b, hi, lo)."""
    k: int
    offsets: np.ndarray   # uint32, n_groups + 1
    value_index: np.ndarray  # uint32
    variant: np.ndarray   # uint8
    amount: np.ndarray    # uint32

    @property
    def n_constraints(self) -> int:
        return (len(self.offsets) - 1) // self.k

    @staticmethod
    def from_lists(constraints, slots) -> "OperandCSR":
        counts, vi, va, am = [], [], [], []
        for c in constraints:
            for name in slots:
                op = getattr(c, name)
                counts.append(len(op))
                for t in op:
                    vi.append(t.value_index)
                    va.append(t.shift_variant)
                    am.append(t.amount)
        offsets = np.zeros(len(counts) + 1, dtype=np.uint32)
        offsets[1:] = np.cumsum(counts, dtype=np.uint64)
        return OperandCSR(len(slots), offsets, np.array(vi, dtype=np.uint32),
                          np.array(va, dtype=np.uint8), np.array(am, dtype=np.uint32))

    def padded(self, n: int) -> "OperandCSR":
        extra = n - self.n_constraints
        if extra <= 0:
            return self
        offsets = np.concatenate([self.offsets, np.full(extra * self.k, self.offsets[-1],
                                                        dtype=np.uint32)])
        return OperandCSR(self.k, offsets, self.value_index, self.variant, self.amount)

    def serialize_into(self, out: bytearray) -> None:
        n = self.n_constraints
        counts = np.diff(self.offsets.astype(np.int64))
        n_groups = len(counts)
        size = 4 + 4 * n_groups + 9 * len(self.value_index)
        buf = np.zeros(size, dtype=np.uint8)
        buf[:4] = np.frombuffer(struct.pack("<I", n), dtype=np.uint8)
        # group g header at 4 + 4*g + 9*offsets[g]; its terms follow
        hdr = 4 + 4 * np.arange(n_groups, dtype=np.int64) + 9 * self.offsets[:-1].astype(np.int64)
        cb = counts.astype(np.uint32).view(np.uint8).reshape(-1, 4)
        for j in range(4):
            buf[hdr + j] = cb[:, j]
        if len(self.value_index):
            grp = np.repeat(np.arange(n_groups), counts)
            pos = 4 + 4 * (grp + 1) + 9 * np.arange(len(self.value_index), dtype=np.int64)
            vb = self.value_index.astype(np.uint32).view(np.uint8).reshape(-1, 4)
            ab = self.amount.astype(np.uint32).view(np.uint8).reshape(-1, 4)
            for j in range(4):
                buf[pos + j] = vb[:, j]
            buf[pos + 4] = self.variant
            for j in range(4):
                buf[pos + 5 + j] = ab[:, j]
        out.extend(buf.tobytes())


@dataclass
class ConstraintSystem:
    layout: ValueVecLayout
    constants: list
    and_constraints: list
    mul_constraints: list
    and_csr: OperandCSR | None = None
    mul_csr: OperandCSR | None = None

    SERIALIZATION_VERSION = 2

    def and_operands(self) -> OperandCSR:
        if self.and_csr is None:
            self.and_csr = OperandCSR.from_lists(self.and_constraints, ("a", "b", "c"))
        return self.and_csr

    def mul_operands(self) -> OperandCSR:
        if self.mul_csr is None:
            self.mul_csr = OperandCSR.from_lists(self.mul_constraints, ("a", "b", "hi", "lo"))
        return self.mul_csr

    def n_and(self) -> int:
        return self.and_operands().n_constraints

    def n_mul(self) -> int:
        return self.mul_operands().n_constraints

    def serialize(self) -> bytes:
        out = bytearray()
        u32 = lambda v: out.extend(struct.pack("<I", v))  # noqa: E731
        u32(self.SERIALIZATION_VERSION)
        L = self.layout
        for v in (L.n_const, L.n_inout, L.n_witness, L.n_internal, L.offset_inout,
                  L.offset_witness, L.committed_total_len, L.n_scratch):
            u32(v)
        u32(len(self.constants))
        for w in self.constants:
            out.extend(struct.pack("<Q", int(w)))
        self.and_operands().serialize_into(out)
        self.mul_operands().serialize_into(out)
        return bytes(out)

    def serialize_lists(self) -> bytes:
        """Reference-order serialization from the constraint objects (cross-check of the CSR
        path)."""
        out = bytearray()
        u32 = lambda v: out.extend(struct.pack("<I", v))  # noqa: E731
        u32(self.SERIALIZATION_VERSION)
        L = self.layout
        for v in (L.n_const, L.n_inout, L.n_witness, L.n_internal, L.offset_inout,
                  L.offset_witness, L.committed_total_len, L.n_scratch):
            u32(v)
        u32(len(self.constants))
        for w in self.constants:
            out.extend(struct.pack("<Q", int(w)))

        def operand(op):
            u32(len(op))
            for t in op:
                u32(t.value_index)
                out.append(t.shift_variant)
                u32(t.amount)

        u32(len(self.and_constraints))
        for c in self.and_constraints:
            operand(c.a), operand(c.b), operand(c.c)
        u32(len(self.mul_constraints))
        for c in self.mul_constraints:
            operand(c.a), operand(c.b), operand(c.hi), operand(c.lo)
        return bytes(out)

    @classmethod
    def deserialize(cls, data: bytes) -> "ConstraintSystem":
        """ConstraintSystem::deserialize (constraint_system.rs:617-650): version 2, the layout, the
        constants (their count must equal n_const), then the AND and MUL constraint lists."""
        pos = 0

        def take(n):
            nonlocal pos
            if pos + n > len(data):
                raise ValueError("NotEnoughBytes")
            b = data[pos:pos + n]
            pos += n
            return b

        u32 = lambda: struct.unpack("<I", take(4))[0]  # noqa: E731
        if u32() != cls.SERIALIZATION_VERSION:
            raise ValueError("InvalidConstruction: ConstraintSystem::version")
        layout = ValueVecLayout(*[u32() for _ in range(8)])
        constants = [struct.unpack("<Q", take(8))[0] for _ in range(u32())]
        if len(constants) != layout.n_const:
            raise ValueError("InvalidConstruction: ConstraintSystem::constants")

        def operand():
            out = []
            for _ in range(u32()):
                vi = u32()
                variant = take(1)[0]
                amount = u32()
                if variant > ROTR32:
                    raise ValueError("UnknownEnumVariant: ShiftVariant")
                out.append(ShiftedValueIndex(vi, variant, amount))
            return out

        ands = [AndConstraint(operand(), operand(), operand()) for _ in range(u32())]
        muls = [MulConstraint(operand(), operand(), operand(), operand()) for _ in range(u32())]
        return cls(layout, constants, ands, muls)

    def prepared(self) -> "ConstraintSystem":
        """validate_and_prepare: pad the constraint lists to powers of two (>= 8 AND, >= 1 MUL)."""
        n_and = max(MIN_AND_CONSTRAINTS, self.n_and())
        n_and = 1 << (n_and - 1).bit_length()
        n_mul = max(MIN_MUL_CONSTRAINTS, self.n_mul())
        n_mul = 1 << (n_mul - 1).bit_length()
        return ConstraintSystem(self.layout, list(self.constants), [], [],
                                self.and_operands().padded(n_and), self.mul_operands().padded(n_mul))


def shifted(words: np.ndarray, variant: int, amount: int) -> np.ndarray:
    """eval_shifted_word (verifier/core/src/verify.rs:14-26) on a numpy uint64 array."""
    w = words.astype(np.uint64)
    n = np.uint64(amount)
    if variant == SLL:
        return w << n
    if variant == SLR:
        return w >> n
    if variant == SAR:
        return (w.view(np.int64) >> np.int64(amount)).view(np.uint64)
    if variant == ROTR:
        return w if amount == 0 else ((w >> n) | (w << np.uint64(64 - amount)))
    lo = (w & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    hi = (w >> np.uint64(32)).astype(np.uint32)
    s = np.uint32(amount & 31)
    if variant == SLL32:
        lo2, hi2 = lo << s, hi << s
    elif variant == SRL32:
        lo2, hi2 = lo >> s, hi >> s
    elif variant == SRA32:
        lo2 = (lo.view(np.int32) >> np.int32(amount & 31)).view(np.uint32)
        hi2 = (hi.view(np.int32) >> np.int32(amount & 31)).view(np.uint32)
    else:  # ROTR32
        if amount & 31 == 0:
            lo2, hi2 = lo, hi
        else:
            r = np.uint32(32 - (amount & 31))
            lo2, hi2 = (lo >> s) | (lo << r), (hi >> s) | (hi << r)
    return (hi2.astype(np.uint64) << np.uint64(32)) | lo2.astype(np.uint64)


def eval_operand(values: np.ndarray, operand) -> int:
    acc = np.uint64(0)
    for t in operand:
        acc ^= shifted(values[t.value_index:t.value_index + 1], t.shift_variant, t.amount)[0]
    return int(acc)


def operand_words(values: np.ndarray, operands) -> np.ndarray:
    """eval_operand for a list of operands -> uint64 array."""
    return np.array([eval_operand(values, op) for op in operands], dtype=np.uint64)


@dataclass
class SyntheticCircuit:
    cs: ConstraintSystem
    witness: np.ndarray  # committed_total_len uint64 words


def _random_term_arrays(rng, n, pool_lo, pool_hi, max_terms):
    """Operand terms as arrays: (n, max_terms) value indices / variants / amounts and a count."""
    counts = rng.integers(1, max_terms + 1, size=n)
    idx = rng.integers(pool_lo, pool_hi, size=(n, max_terms))
    variant = rng.integers(0, 8, size=(n, max_terms))
    amount = np.where(variant >= 4, rng.integers(0, 32, size=(n, max_terms)),
                      rng.integers(0, 64, size=(n, max_terms)))
    # canonical form: a zero shift is always Sll (validate(), constraint_system.rs:494-500)
    variant = np.where(amount == 0, SLL, variant)
    return idx, variant, amount, counts


def shifted_by(words: np.ndarray, variant: int, amounts: np.ndarray) -> np.ndarray:
    """shifted() with a per-word shift amount (same variant for all words)."""
    w = words.astype(np.uint64)
    a = amounts.astype(np.uint64)
    if variant == SLL:
        return w << a
    if variant == SLR:
        return w >> a
    if variant == SAR:
        return (w.view(np.int64) >> a.astype(np.int64)).view(np.uint64)
    if variant == ROTR:
        rot = (w >> a) | (w << ((np.uint64(64) - a) & np.uint64(63)))
        return np.where(a == 0, w, rot)
    lo = (w & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    hi = (w >> np.uint64(32)).astype(np.uint32)
    s = (a & np.uint64(31)).astype(np.uint32)
    if variant == SLL32:
        lo2, hi2 = lo << s, hi << s
    elif variant == SRL32:
        lo2, hi2 = lo >> s, hi >> s
    elif variant == SRA32:
        si = s.astype(np.int32)
        lo2 = (lo.view(np.int32) >> si).view(np.uint32)
        hi2 = (hi.view(np.int32) >> si).view(np.uint32)
    else:  # ROTR32
        r = (np.uint32(32) - s) & np.uint32(31)
        lo2 = np.where(s == 0, lo, (lo >> s) | (lo << r))
        hi2 = np.where(s == 0, hi, (hi >> s) | (hi << r))
    return (hi2.astype(np.uint64) << np.uint64(32)) | lo2.astype(np.uint64)


def _eval_term_arrays(values, idx, variant, amount, counts):
    n, m = idx.shape
    acc = np.zeros(n, dtype=np.uint64)
    for j in range(m):
        active = counts > j
        w = values[idx[:, j]]
        res = np.zeros(n, dtype=np.uint64)
        for v in range(8):
            for_v = (variant[:, j] == v) & active
            if for_v.any():
                res[for_v] = shifted_by(w[for_v], v, amount[for_v, j])
        acc ^= res
    return acc


def _terms_to_lists(idx, variant, amount, counts):
    out = []
    for i in range(idx.shape[0]):
        out.append([ShiftedValueIndex(int(idx[i, j]), int(variant[i, j]), int(amount[i, j]))
                    for j in range(int(counts[i]))])
    return out


def synthetic_circuit(log_committed_words: int, n_and: int, n_mul: int = 1, seed: int = 0,
                      n_layers: int = 4, max_terms: int = 3, log_public: int = 1,
                      n_const: int = 1) -> SyntheticCircuit:
    """A satisfiable circuit with 2^log_committed_words committed words.

    Layout: [constants | inout | padding] (2^log_public words, the public segment), then random
    witness inputs, then one internal word per AND constraint and two (lo, hi) per MUL.  AND
    constraints come in `n_layers` layers whose operands read earlier words; c = w_new ^ extra terms
    with w_new chosen so that (A & B) ^ C = 0.
    """
    rng = np.random.default_rng(seed)
    total = 1 << log_committed_words
    offset_witness = 1 << log_public
    n_inout = offset_witness - n_const
    n_internal = n_and + 2 * n_mul
    n_witness = total - offset_witness - n_internal
    if n_witness < 1:
        raise ValueError("too many constraints for the committed length")
    values = np.zeros(total, dtype=np.uint64)
    values[:n_const] = rng.integers(0, _M64, size=n_const, dtype=np.uint64, endpoint=True)
    values[n_const:offset_witness] = rng.integers(0, _M64, size=n_inout, dtype=np.uint64, endpoint=True)
    w0 = offset_witness
    values[w0:w0 + n_witness] = rng.integers(0, _M64, size=n_witness, dtype=np.uint64, endpoint=True)
    next_internal = w0 + n_witness
    per_layer = [n_and // n_layers + (1 if i < n_and % n_layers else 0) for i in range(n_layers)]
    pool_hi = next_internal
    and_parts = []  # per layer: (term arrays of a, b, c) with counts
    for layer_n in per_layer:
        if layer_n == 0:
            continue
        ia, va, aa, ca = _random_term_arrays(rng, layer_n, 0, pool_hi, max_terms)
        ib, vb, ab, cb = _random_term_arrays(rng, layer_n, 0, pool_hi, max_terms)
        ic, vc, ac, _ = _random_term_arrays(rng, layer_n, 0, pool_hi, max_terms - 1)
        cc = rng.integers(0, max_terms, size=layer_n)  # extra c terms (0..max_terms-1)
        A = _eval_term_arrays(values, ia, va, aa, ca)
        B = _eval_term_arrays(values, ib, vb, ab, cb)
        extra = (_eval_term_arrays(values, ic, vc, ac, cc) if ic.shape[1]
                 else np.zeros(layer_n, np.uint64))
        new_idx = np.arange(next_internal, next_internal + layer_n)
        values[new_idx] = (A & B) ^ extra
        # c = plain(new word) followed by the extra terms
        ic2 = np.concatenate([new_idx[:, None], ic], axis=1)
        vc2 = np.concatenate([np.zeros((layer_n, 1), dtype=vc.dtype), vc], axis=1)
        ac2 = np.concatenate([np.zeros((layer_n, 1), dtype=ac.dtype), ac], axis=1)
        and_parts.append(((ia, va, aa, ca), (ib, vb, ab, cb), (ic2, vc2, ac2, cc + 1)))
        next_internal += layer_n
        pool_hi = next_internal
    mul_parts = []
    if n_mul:
        ia, va, aa, ca = _random_term_arrays(rng, n_mul, 0, pool_hi, max_terms)
        ib, vb, ab, cb = _random_term_arrays(rng, n_mul, 0, pool_hi, max_terms)
        A = _eval_term_arrays(values, ia, va, aa, ca)
        B = _eval_term_arrays(values, ib, vb, ab, cb)
        hi_idx = np.zeros((n_mul, 1), dtype=np.int64)
        lo_idx = np.zeros((n_mul, 1), dtype=np.int64)
        for i in range(n_mul):
            prod = int(A[i]) * int(B[i])
            lo_i, hi_i = next_internal, next_internal + 1
            values[lo_i] = np.uint64(prod & 0xFFFFFFFFFFFFFFFF)
            values[hi_i] = np.uint64(prod >> 64)
            lo_idx[i, 0], hi_idx[i, 0] = lo_i, hi_i
            next_internal += 2
        zero = np.zeros((n_mul, 1), dtype=np.int64)
        one = np.ones(n_mul, dtype=np.int64)
        mul_parts.append(((ia, va, aa, ca), (ib, vb, ab, cb), (hi_idx, zero, zero, one),
                          (lo_idx, zero, zero, one)))
    layout = ValueVecLayout(n_const=n_const, n_inout=n_inout, n_witness=n_witness,
                            n_internal=n_internal, offset_inout=n_const,
                            offset_witness=offset_witness, committed_total_len=total)
    cs = ConstraintSystem(layout, [int(x) for x in values[:n_const]], [], [],
                          _csr_from_parts(and_parts, 3), _csr_from_parts(mul_parts, 4))
    return SyntheticCircuit(cs, values)


def _csr_from_parts(parts, k: int) -> OperandCSR:
    """Interleave per-slot term arrays (constraint-major, slot-minor) into one CSR."""
    counts_all, vi_all, va_all, am_all = [], [], [], []
    for slots in parts:
        n = slots[0][0].shape[0]
        counts = np.stack([s[3] for s in slots], axis=1).reshape(-1)  # (n*k,)
        width = max(s[0].shape[1] for s in slots)
        idx = np.zeros((n, k, width), dtype=np.int64)
        var = np.zeros((n, k, width), dtype=np.int64)
        amt = np.zeros((n, k, width), dtype=np.int64)
        for j, s in enumerate(slots):
            w = s[0].shape[1]
            idx[:, j, :w], var[:, j, :w], amt[:, j, :w] = s[0], s[1], s[2]
        mask = np.arange(width)[None, None, :] < np.stack([s[3] for s in slots], axis=1)[:, :, None]
        counts_all.append(counts)
        vi_all.append(idx[mask])
        va_all.append(var[mask])
        am_all.append(amt[mask])
    if not parts:
        return OperandCSR(k, np.zeros(1, dtype=np.uint32), np.zeros(0, np.uint32),
                          np.zeros(0, np.uint8), np.zeros(0, np.uint32))
    counts = np.concatenate(counts_all)
    offsets = np.zeros(len(counts) + 1, dtype=np.uint32)
    offsets[1:] = np.cumsum(counts)
    return OperandCSR(k, offsets, np.concatenate(vi_all).astype(np.uint32),
                      np.concatenate(va_all).astype(np.uint8),
                      np.concatenate(am_all).astype(np.uint32))


def csr_operand(csr: OperandCSR, group: int):
    lo, hi = int(csr.offsets[group]), int(csr.offsets[group + 1])
    return [ShiftedValueIndex(int(csr.value_index[t]), int(csr.variant[t]), int(csr.amount[t]))
            for t in range(lo, hi)]


def eval_operands_csr(values: np.ndarray, csr: OperandCSR) -> np.ndarray:
    """All operands of a CSR list -> (n_constraints, k) uint64 (vectorized eval_operand)."""
    counts = np.diff(csr.offsets.astype(np.int64))
    n_groups = len(counts)
    grp = np.repeat(np.arange(n_groups), counts)
    w = values[csr.value_index.astype(np.int64)]
    res = np.zeros(len(w), dtype=np.uint64)
    for v in range(8):
        for a in np.unique(csr.amount[csr.variant == v]) if len(w) else []:
            sel = (csr.variant == v) & (csr.amount == a)
            res[sel] = shifted(w[sel], v, int(a))
    out = np.zeros(n_groups, dtype=np.uint64)
    np.bitwise_xor.at(out, grp, res)
    return out.reshape(-1, csr.k)


def check_satisfied(cs: ConstraintSystem, values: np.ndarray) -> bool:
    """verify_constraints (verifier/core/src/verify.rs:74-100)."""
    for i, k in enumerate(cs.constants):
        if int(values[i]) != int(k):
            return False
    abc = eval_operands_csr(values, cs.and_operands())
    if np.any((abc[:, 0] & abc[:, 1]) ^ abc[:, 2]):
        return False
    m = eval_operands_csr(values, cs.mul_operands())
    for a, b, hi, lo in m:
        prod = int(a) * int(b)
        if int(lo) != prod & 0xFFFFFFFFFFFFFFFF or int(hi) != prod >> 64:
            return False
    return True
