"""Independent pure-Python big-integer model of the CKKS residue math.

Written from the mathematical definitions (negacyclic ring Z_q[X]/(X^N+1),
CRT basis conversion, floor rescale), not from the oracle's code, so that it
can cross-check the C++ oracle on small rings.  Slow by design: small N only.
"""
from functools import reduce


def bitrev(x, bits):
    return int(format(x, "0%db" % bits)[::-1], 2) if bits else 0


def negacyclic_mul(a, b, q):
    """Schoolbook product in Z_q[X]/(X^N+1)."""
    n = len(a)
    out = [0] * n
    for i, ai in enumerate(a):
        if ai == 0:
            continue
        for j, bj in enumerate(b):
            t = i + j
            if t < n:
                out[t] += ai * bj
            else:
                out[t - n] -= ai * bj
    return [v % q for v in out]


def ntt_closed_form(a, q, psi):
    """Position p holds a(psi^(2*bitrev(p)+1)) — the reference transform's order."""
    n = len(a)
    lg = n.bit_length() - 1
    out = []
    for p in range(n):
        ev = pow(psi, 2 * bitrev(p, lg) + 1, q)
        acc, pw = 0, 1
        for c in a:
            acc += c * pw
            pw = pw * ev % q
        out.append(acc % q)
    return out


def prod(xs):
    return reduce(lambda u, v: u * v, xs, 1)


def modup(xq, qs, bs, level):
    """B_j = sum_i [x_i (Q_l/q_i)^-1]_{q_i} (Q_l/q_i) mod b_j, i <= level (no correction)."""
    Ql = prod(qs[: level + 1])
    n = len(xq[0])
    out = []
    for b in bs:
        row = []
        for c in range(n):
            acc = 0
            for i in range(level + 1):
                qi = qs[i]
                hat = Ql // qi
                y = xq[i][c] * pow(hat % qi, -1, qi) % qi
                acc += y * hat
            row.append(acc % b)
        out.append(row)
    return out


def moddown(xq, xb, qs, bs, level):
    """out_i = (x_i - sum_j [x_j (B/b_j)^-1]_{b_j} (B/b_j)) * B^-1 mod q_i."""
    Bp = prod(bs)
    n = len(xq[0])
    out = []
    for i in range(level + 1):
        qi = qs[i]
        row = []
        for c in range(n):
            acc = 0
            for j, b in enumerate(bs):
                hat = Bp // b
                acc += (xb[j][c] * pow(hat % b, -1, b) % b) * hat
            row.append((xq[i][c] - acc) * pow(Bp % qi, -1, qi) % qi)
        out.append(row)
    return out


def rescale(x, qs, level):
    """Floor rescale: (x_i - x_level) * q_level^-1 mod q_i for i < level."""
    ql = qs[level]
    return [[(x[i][c] - x[level][c]) * pow(ql % qs[i], -1, qs[i]) % qs[i] for c in range(len(x[0]))]
            for i in range(level)]


def automorph(a, power, q):
    """a(X) -> a(X^power) in Z_q[X]/(X^N+1)."""
    n = len(a)
    out = [0] * n
    for i, c in enumerate(a):
        t = i * power % (2 * n)
        if t >= n:
            out[t - n] = (-c) % q
        else:
            out[t] = c % q
    return out
