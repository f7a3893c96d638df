"""Coefficient-adjusted CRT focuses and canonical coordinate tiles.

Mirrors pseudocube/focus.py:11-191 (constants, factors, Focus, Config, Tile,
targeted_coordinates).  x = uB - vA with coprime focus moduli A, B; the constraints of primes
dividing A are carried by u (residues multiplied by B^-1), those of primes dividing B by v
(residues multiplied by (-A)^-1); every other prime <= p is a residual filter on x.  The
canonical pair has 0 <= v < B.
"""
from __future__ import annotations

from dataclasses import dataclass
from math import gcd, prod
from typing import Any, Iterator

from .predicate import validate_p
from .tables import allowed, definition, sieve_primes

A619 = 701856356111039402
B619 = 693110504329192503
MAX = (1 << 64) - 1


def factors(n: int, p: int) -> list[int]:
    """Prime-power ring moduli of a focus modulus: squarefree primes and at most one full 9."""
    if not 1 <= n < 1 << 63:
        raise ValueError('focus modulus must be positive and below 2^63')
    rings: list[int] = []
    for q in sieve_primes(p):
        if n % q:
            continue
        power = 1
        while n % q == 0:
            n //= q
            power *= q
        if power != (9 if q == 3 else q):
            raise ValueError('only squarefree primes and one complete factor 9 are supported')
        rings.append(power)
    if n != 1:
        raise ValueError('focus contains a prime above the active cutoff')
    return rings


@dataclass(frozen=True)
class Focus:
    """Allowed residues of one focus modulus, ring by ring (ascending ring moduli)."""
    modulus: int
    rings: tuple[tuple[int, tuple[int, ...]], ...]

    @property
    def count(self) -> int:
        return prod(len(residues) for _, residues in self.rings)

    @property
    def terms(self) -> tuple[tuple[int, ...], ...]:
        """CRT basis terms a * (M/q) * ((M/q)^-1 mod q) mod M of every allowed residue a."""
        M = self.modulus
        out = []
        for q, residues in self.rings:
            cofactor = M // q
            basis = cofactor * pow(cofactor, -1, q) % M
            out.append(tuple(a * basis % M for a in residues))
        return tuple(out)

    def at(self, index: int) -> int:
        """Mixed-radix index (ring 0 fastest) to focus value in [0, M)."""
        if not 0 <= index < self.count:
            raise ValueError('focus index out of bounds')
        value = 0
        for terms in self.terms:
            index, digit = divmod(index, len(terms))
            value = (value + terms[digit]) % self.modulus
        return value

    def rank(self, coordinate: int) -> tuple[int, int]:
        period, value = divmod(coordinate, self.modulus)
        index, radix = 0, 1
        for q, residues in self.rings:
            index += residues.index(value % q) * radix
            radix *= len(residues)
        return period, index

    def indices(self, start: int, end: int, period: int = 0) -> Iterator[int]:
        if not 0 <= start <= end <= self.count or period < 0:
            raise ValueError('invalid focus index interval')
        for index in range(start, end):
            yield period * self.modulus + self.at(index)

    def contains(self, y: int) -> bool:
        return y >= 0 and all(y % q in residues for q, residues in self.rings)

    def halves(self) -> tuple[tuple[tuple[int, ...], ...], tuple[tuple[int, ...], ...]]:
        """Balanced two-way split of the ring terms (pseudocube/focus.py:81-87)."""
        terms = self.terms
        sizes = [len(t) for t in terms]

        def worst(mask: int) -> int:
            inside = prod(s for i, s in enumerate(sizes) if mask >> i & 1)
            return max(inside, prod(sizes) // inside)

        best = min(range(1 << len(terms)), key=worst)
        return (tuple(t for i, t in enumerate(terms) if best >> i & 1),
                tuple(t for i, t in enumerate(terms) if not best >> i & 1))


@dataclass(frozen=True)
class Config:
    p: int
    lo: int
    hi: int
    A: int
    B: int

    def __post_init__(self) -> None:
        validate_p(self.p)
        if not 0 <= self.lo < self.hi <= 3 * 10**27 or gcd(self.A, self.B) != 1:
            raise ValueError('invalid interval, arithmetic bound, or coprimality')
        factors(self.A, self.p)
        factors(self.B, self.p)
        maximum_u = (self.hi + (self.B - 1) * self.A) // self.B
        if maximum_u > MAX or maximum_u * self.B >= 1 << 128:
            raise ValueError('intermediates exceed implementation bounds')

    def focuses(self) -> tuple[Focus, Focus]:
        built = []
        for modulus, coefficient in ((self.A, self.B), (self.B, -self.A)):
            rings = []
            for q in factors(modulus, self.p):
                inverse = pow(coefficient, -1, q)
                rings.append((q, tuple(sorted({a * inverse % q for a in allowed(q)}))))
            built.append(Focus(modulus, tuple(rings)))
        return built[0], built[1]

    def canonical(self, n: int) -> tuple[int, int]:
        v = (-n * pow(self.A, -1, self.B)) % self.B if self.B > 1 else 0
        return (n + v * self.A) // self.B, v

    def u_interval(self, v: int) -> tuple[int, int]:
        """Exact half-open u range with lo < uB - vA <= hi."""
        return (self.lo + v * self.A) // self.B + 1, (self.hi + v * self.A) // self.B + 1

    def coverage(self) -> dict[str, str]:
        af, bf = factors(self.A, self.p), factors(self.B, self.p)
        where = {}
        for q in (9, *sieve_primes(self.p)):
            if q == 3:
                continue
            where[str(q)] = 'A_focus' if q in af else 'B_focus' if q in bf else 'residual'
        where['3'] = 'mod9'
        return where

    def residuals(self) -> list[int]:
        return [int(q) for q, location in self.coverage().items() if location == 'residual']

    def filter_order(self) -> list[int]:
        """Residual filters in execution order: 9, then q = 1 mod 3, then the rest, each ascending
        (pseudocube/gpu.py:134, pseudocube/batch_experiment.py:84-86)."""
        return sorted(self.residuals(), key=lambda q: (q != 9 and q % 3 != 1, q))

    def filter_groups(self) -> list[list[int]]:
        order = self.filter_order()
        return [order[i:i + 4] for i in range(0, len(order), 4)]

    def manifest(self) -> dict[str, Any]:
        af, bf = self.focuses()
        maximum_u = (self.hi + (self.B - 1) * self.A) // self.B
        return dict(schema_version=1, search_type='pseudocube', p=self.p, lo_exclusive=str(self.lo),
                    hi_inclusive=str(self.hi), A=str(self.A), B=str(self.B), canonical='v-in-[0,B)',
                    coverage=self.coverage(), table_sha256=definition(self.p)['sha256'],
                    focus_counts=[str(af.count), str(bf.count)],
                    arithmetic_bounds=dict(max_u=str(maximum_u), max_v=str(self.B - 1),
                                           max_uB=str(maximum_u * self.B), max_vA=str((self.B - 1) * self.A),
                                           x_bits=self.hi.bit_length(),
                                           product_bits=(maximum_u * self.B).bit_length()))


@dataclass(frozen=True)
class Tile:
    first: int
    end: int

    def validate(self, config: Config) -> None:
        if not 0 <= self.first < self.end <= config.B:
            raise ValueError('tile must be a nonempty canonical v interval')

    def envelope(self, config: Config) -> dict[str, str]:
        self.validate(config)
        u_min = config.u_interval(self.first)[0]
        u_max = config.u_interval(self.end - 1)[1] - 1
        return dict(u_min=str(u_min), u_max=str(u_max), v_min=str(self.first), v_max=str(self.end - 1),
                    x_min=str(u_min * config.B - (self.end - 1) * config.A),
                    x_max=str(u_max * config.B - self.first * config.A))

    def split(self) -> tuple['Tile', 'Tile']:
        if self.end - self.first < 2:
            raise ValueError('unsplittable tile')
        middle = (self.first + self.end) // 2
        return Tile(self.first, middle), Tile(middle, self.end)

    def manifest(self, config: Config) -> dict[str, Any]:
        return dict(kind='v-window', first=str(self.first), end=str(self.end), envelope=self.envelope(config))


def targeted_coordinates(config: Config, n: int, radius: int = 1) -> tuple[list[int], list[int]]:
    """CRT index neighbourhoods around n's canonical pair; n itself is never injected."""
    u, v = config.canonical(n)
    af, bf = config.focuses()
    period, ui = af.rank(u)
    vp, vi = bf.rank(v)
    if vp != 0:
        raise ValueError('noncanonical v')
    return (list(af.indices(max(0, ui - radius), min(af.count, ui + radius + 1), period)),
            list(bf.indices(max(0, vi - radius), min(bf.count, vi + radius + 1))))
