"""CPU emulation of the warp-per-cell kernel's schedules (test infrastructure).

kppcu writes, into each mechanism's header, the tables that the warp-per-cell
kernel (kpp_b200/csrc/kpp_coop.cuh) stages in shared memory: the product
factors and weights of Fun and Jac_SP, the lane streams of the Vdot and
Jacobian sums, and the iteration counts and lane streams of the LU
factorisation and of the forward substitution (the backward substitution
runs on one lane as the header's straight-line kpp_solve_bw, restated here
row by row in KppSolve's order).  This module
reads those tables back from the header and executes them the way the kernel
does -- iteration by iteration, lane by lane, in IEEE double arithmetic -- so
that tests can require the results to equal the reference's own generated
Fun, Jac_SP, KppDecomp and KppSolve bit for bit.  Lanes within one iteration
never touch what another lane of the same iteration writes, so running them
one after the other gives what the warp computes.
"""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np

LANES = 32
NOP = 0xFFFFFFFF


class CoopTables:
    def __init__(self, header: Path):
        text = Path(header).read_text()
        if "#define KPP_COOP 1" not in text:
            raise ValueError(f"{header}: no warp-per-cell tables")
        body = text[text.index("namespace kpp_coop {"):text.index("}  // namespace kpp_coop")]
        self.c = {k: int(v) for k, v in re.findall(r"(\w+) = (-?\d+)", body)
                  if not k.startswith("__")}
        self.tab = self._array(body, "tab", int)
        # the kernel stages NKC constants: an index beyond them must fail here too
        self.kc = self._array(body, "kc", float)[: self.c["NKC"]]
        self.nvar = int(re.search(r"#define KPP_NVAR (\d+)", text).group(1))
        self.nfix = int(re.search(r"#define KPP_NFIX_TRUE (\d+)", text).group(1))
        self.lu_nz = int(re.search(r"#define KPP_LU_NONZERO (\d+)", text).group(1))

    @staticmethod
    def _array(body, name, conv):
        m = re.search(name + r"\[\d+\] = \{([^}]*)\}", body)
        vals = [v.strip() for v in m.group(1).split(",") if v.strip()]
        return [conv(v) for v in vals]

    def __getattr__(self, k):
        try:
            return self.__dict__["c"][k]
        except KeyError:
            raise AttributeError(k) from None

    # -- products and sums ----------------------------------------------------
    def weights(self, off, rounds, rc):
        rb = self.RATE_BITS
        out = []
        for t in range(rounds * LANES):
            w = self.tab[off + t]
            rct, k1, k2 = w & ((1 << rb) - 1), (w >> rb) & 4095, (w >> (rb + 12)) & 4095
            base = rc[rct] if rct != self.NO_RATE else self.kc[k1]
            out.append(base * self.kc[k2])
        return out

    def products(self, off_f, weights, n, vext):
        out = [0.0] * n
        for t in range(n):
            f = self.tab[off_f + t]
            v = weights[t]
            for k in range(4):
                v = v * vext[(f >> (8 * k)) & 255]
            out[t] = v
        return out

    def sums(self, off, per_lane, src, nout, neg, ghinv=None):
        sb, cb = self.SUM_SRC_BITS, self.SUM_COEF_BITS
        fb = sb + cb
        out = [None] * nout
        for lane in range(LANES):
            acc = 0.0
            for k in range(per_lane):
                e = self.tab[off + k * LANES + lane]
                if e == NOP:
                    continue
                start, end = (e >> fb) & 1, (e >> (fb + 1)) & 1
                zero, diag = (e >> (fb + 2)) & 1, (e >> (fb + 3)) & 1
                dst = e >> (fb + 4)
                if zero:
                    val = -0.0 if neg else 0.0
                else:
                    p = self.kc[(e >> sb) & ((1 << cb) - 1)] * src[e & ((1 << sb) - 1)]
                    acc = p if start else acc + p
                    val = -acc if neg else acc
                if end:
                    if diag and ghinv is not None:
                        val = val + ghinv
                    out[dst] = val
        return out

    def fun(self, var, fix, rc):
        vext = list(var) + list(fix[: self.nfix]) + [1.0]
        a = self.products(self.O_PF, self.weights(self.O_WF, self.RF, rc), self.NA, vext)
        return self.sums(self.O_SV, self.LV, a, self.nvar, neg=False)

    def jac(self, var, fix, rc, neg=False, ghinv=None):
        vext = list(var) + list(fix[: self.nfix]) + [1.0]
        b = self.products(self.O_PJ, self.weights(self.O_WJ, self.RJ, rc), self.NB, vext)
        return self.sums(self.O_SJ, self.LJ, b, self.lu_nz, neg=neg, ghinv=ghinv)

    # -- iterated phases ------------------------------------------------------
    def _iterate(self, off_c, off_s, iters, step):
        pos = [0] * LANES
        for it in range(iters):
            for lane in range(LANES):
                n = (self.tab[off_c + it * 4 + lane // 8] >> (4 * (lane % 8))) & 15
                for _ in range(n):
                    step(lane, self.tab[off_s + pos[lane] * LANES + lane])
                    pos[lane] += 1

    def decomp(self, jvs):
        """In place; returns k+1 for the first row whose diagonal is zero on
        entry to its elimination (its original value), else 0."""
        j = jvs
        diag = self.tab[self.O_DIAG:self.O_DIAG + self.nvar]
        for k in range(self.nvar):
            if j[diag[k]] == 0.0:
                return k + 1
        b = self.LU_BITS
        mask = (1 << b) - 1

        def step(lane, e):
            t, m, s = (e >> (2 * b)) & mask, (e >> b) & mask, e & mask
            if e >> 31:
                j[t] = j[t] / j[s]
            else:
                j[t] = j[t] + (-j[m]) * j[s]

        self._iterate(self.O_CLU, self.O_LU, self.IT_LU, step)
        return 0

    def solve(self, jvs, x, lu_pattern):
        """(LU) x = b in place, b given in x: the forward substitution from the
        tables, then the backward one in KppSolve's order (src/gen.c:1960-2034:
        each row's terms left to right, then the division by the diagonal) over
        lu_pattern = (LU_IROW, LU_ICOL, LU_CROW, LU_DIAG)."""
        b, c = self.LU_BITS, self.X_BITS
        acc = [0.0] * LANES

        def step(lane, e):
            a, cc = e & ((1 << b) - 1), (e >> b) & ((1 << c) - 1)
            r = (e >> (b + c)) & ((1 << c) - 1)
            f = b + 2 * c
            if (e >> f) & 1:
                acc[lane] = x[r]
            acc[lane] = acc[lane] - jvs[a] * x[cc]
            if (e >> (f + 1)) & 1:
                x[r] = acc[lane]

        self._iterate(self.O_CFW, self.O_FW, self.IT_FW, step)
        _, icol, crow, diag = lu_pattern
        for i in range(self.nvar - 1, -1, -1):
            v = x[i]
            for j in range(diag[i] + 1, crow[i + 1]):
                v = v - jvs[j] * x[icol[j]]
            x[i] = v / jvs[diag[i]]
