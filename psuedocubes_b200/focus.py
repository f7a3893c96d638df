"""Focus moduli, coefficient-adjusted residue rings and canonical v tiles.

The arithmetic is the reference's mathematical contract (docs/mathematics.md:11-44 of the
reference project):

* x = uB - vA with coprime focus moduli A and B.  A prime-power ring q dividing A constrains
  u mod q to B^-1 C_q, a ring dividing B constrains v mod q to (-A)^-1 C_q, where C_q is the set
  of allowed residues of x mod q ({1, 8} for q = 9, the nonzero residues for q = 2 mod 3, the
  nonzero cubic residues for q = 1 mod 3).  Every other prime <= p is a residual filter on x; 3
  is covered by the complete factor 9 and never by two factors of 3.
* Every x has exactly one canonical pair with 0 <= v < B: v = -x A^-1 mod B, u = (x + vA) / B.
* For fixed v, lo < uB - vA <= hi exactly when floor((lo + vA)/B) + 1 <= u < floor((hi + vA)/B) + 1.
* Pairwise coprime ring moduli make the mixed-radix digit tuples (ring 0 fastest) a bijection
  onto the allowed residues mod the focus modulus (the CRT): digit d_q selects a residue r_q and
  the value is sum r_q e_q mod M with the idempotents e_q = (M/q) ((M/q)^-1 mod q).
* u <= floor((hi + (B - 1) A) / B) must fit 64 bits and u B must stay below 2^128.

Public names, arguments, manifest keys and exception types are those of the reference's
pseudocube/focus.py (Config, Focus, Tile, factors, targeted_coordinates), so its callers, its
manifests and the hashes over them see the same values.
"""
from __future__ import annotations

from dataclasses import dataclass
from functools import cached_property
from math import gcd, prod
from typing import Any, Iterator

from .predicate import validate_p
from .tables import allowed, definition, sieve_primes

A619 = 701856356111039402
B619 = 693110504329192503
MAX = (1 << 64) - 1
X_CEILING = 3 * 10**27                  # largest hi the implementation's bounds are checked for

_SQUAREFREE = 'only squarefree primes and one complete factor 9 are supported'


def factors(n: int, p: int) -> list[int]:
    """Ring moduli of the focus modulus n over the primes <= p, ascending: every prime q != 3 that
    divides n exactly once, and 9 when 3 divides n exactly twice."""
    if not 1 <= n < 1 << 63:
        raise ValueError('focus modulus must be positive and below 2^63')
    rings: list[int] = []
    rest = n
    for q in sieve_primes(p):
        if rest == 1:
            break
        if rest % q:
            continue
        ring = 9 if q == 3 else q
        if rest % ring:                                   # 3 without a second factor 3
            raise ValueError(_SQUAREFREE)
        rest //= ring
        if rest % q == 0:                                 # q^2, or 27
            raise ValueError(_SQUAREFREE)
        rings.append(ring)
    if rest != 1:
        raise ValueError('focus contains a prime above the active cutoff')
    return rings


@dataclass(frozen=True)
class Focus:
    """The allowed residues of one focus modulus, ring by ring (ascending ring moduli)."""
    modulus: int
    rings: tuple[tuple[int, tuple[int, ...]], ...]

    @cached_property
    def _idempotents(self) -> tuple[int, ...]:
        """e_q = 1 mod q and 0 mod every other ring of the modulus."""
        M = self.modulus
        return tuple((M // q) * pow(M // q, -1, q) % M for q, _ in self.rings)

    @cached_property
    def _sizes(self) -> tuple[int, ...]:
        return tuple(len(residues) for _, residues in self.rings)

    @cached_property
    def _digit_of(self) -> tuple[dict[int, int], ...]:
        return tuple({r: d for d, r in enumerate(residues)} for _, residues in self.rings)

    @property
    def count(self) -> int:
        return prod(self._sizes)

    @property
    def terms(self) -> tuple[tuple[int, ...], ...]:
        """Per ring, r e_q mod M for every allowed residue r (the CRT basis terms)."""
        M = self.modulus
        return tuple(tuple(r * e % M for r in residues) for (_, residues), e in zip(self.rings, self._idempotents))

    def _digits(self, index: int) -> list[int]:
        digits = []
        for size in self._sizes:
            index, d = divmod(index, size)
            digits.append(d)
        return digits

    def _value(self, digits: list[int]) -> int:
        return sum(residues[d] * e for d, (_, residues), e in zip(digits, self.rings, self._idempotents)) % self.modulus

    def at(self, index: int) -> int:
        """Focus value in [0, M) of a mixed-radix index (ring 0 fastest)."""
        if not 0 <= index < self.count:
            raise ValueError('focus index out of bounds')
        return self._value(self._digits(index))

    def rank(self, coordinate: int) -> tuple[int, int]:
        """(period, index) of a focus coordinate: the inverse of at() within its period."""
        period, value = divmod(coordinate, self.modulus)
        index, radix = 0, 1
        for (q, _), digit_of, size in zip(self.rings, self._digit_of, self._sizes):
            digit = digit_of.get(value % q)
            if digit is None:
                raise ValueError(f'{coordinate} is not in the focus (residue {value % q} mod {q})')
            index += digit * radix
            radix *= size
        return period, index

    def indices(self, start: int, end: int, period: int = 0) -> Iterator[int]:
        """Coordinates period * M + at(i) for i in [start, end), stepping the digits like an
        odometer."""
        if not 0 <= start <= end <= self.count or period < 0:
            raise ValueError('invalid focus index interval')
        if start == end:
            return
        digits = self._digits(start)
        offset = period * self.modulus
        for _ in range(end - start):
            yield offset + self._value(digits)
            for k, size in enumerate(self._sizes):
                digits[k] += 1
                if digits[k] < size:
                    break
                digits[k] = 0

    def contains(self, y: int) -> bool:
        return y >= 0 and all(y % q in digit_of for (q, _), digit_of in zip(self.rings, self._digit_of))

    def halves(self) -> tuple[tuple[tuple[int, ...], ...], tuple[tuple[int, ...], ...]]:
        """The two-way split of the ring terms whose larger side is smallest (the first such
        split in ring-subset order), as the reference's half-sum tables use it."""
        sizes, total = self._sizes, self.count
        best_mask, best = 0, None
        for mask in range(1 << len(sizes)):
            inside = prod(s for k, s in enumerate(sizes) if mask >> k & 1)
            larger = max(inside, total // inside)
            if best is None or larger < best:
                best_mask, best = mask, larger
        terms = self.terms
        return (tuple(t for k, t in enumerate(terms) if best_mask >> k & 1),
                tuple(t for k, t in enumerate(terms) if not best_mask >> k & 1))


def _adjusted(q: int, coefficient: int) -> tuple[int, ...]:
    """Allowed residues of x mod q mapped to the coordinate: r c^-1 mod q for every allowed r."""
    inverse = pow(coefficient, -1, q)
    return tuple(sorted({r * inverse % q for r in allowed(q)}))


@dataclass(frozen=True)
class Config:
    """One search: prime bound p, interval (lo, hi], focus moduli A and B."""
    p: int
    lo: int
    hi: int
    A: int
    B: int

    def __post_init__(self) -> None:
        validate_p(self.p)
        if not 0 <= self.lo < self.hi <= X_CEILING or gcd(self.A, self.B) != 1:
            raise ValueError('invalid interval, arithmetic bound, or coprimality')
        factors(self.A, self.p)
        factors(self.B, self.p)
        if self._max_u() > MAX or self._max_u() * self.B >= 1 << 128:
            raise ValueError('intermediates exceed implementation bounds')

    def _max_u(self) -> int:
        return (self.hi + (self.B - 1) * self.A) // self.B

    def focuses(self) -> tuple[Focus, Focus]:
        """The u focus (rings of A, residues times B^-1) and the v focus (rings of B, residues
        times (-A)^-1)."""
        u_rings = tuple((q, _adjusted(q, self.B)) for q in factors(self.A, self.p))
        v_rings = tuple((q, _adjusted(q, -self.A)) for q in factors(self.B, self.p))
        return Focus(self.A, u_rings), Focus(self.B, v_rings)

    def canonical(self, n: int) -> tuple[int, int]:
        """The canonical pair (u, v) of n, 0 <= v < B."""
        inverse = pow(self.A, -1, self.B) if self.B > 1 else 0
        v = -n * inverse % self.B
        return (n + v * self.A) // self.B, v

    def u_interval(self, v: int) -> tuple[int, int]:
        """Exact half-open u range with lo < uB - vA <= hi."""
        return (self.lo + v * self.A) // self.B + 1, (self.hi + v * self.A) // self.B + 1

    def coverage(self) -> dict[str, str]:
        """Where each constraint is enforced: 'A_focus', 'B_focus', 'residual', and '3': 'mod9'."""
        on_a, on_b = set(factors(self.A, self.p)), set(factors(self.B, self.p))
        where = {}
        for q in (9, *(q for q in sieve_primes(self.p) if q != 3)):
            where[str(q)] = 'A_focus' if q in on_a else 'B_focus' if q in on_b else 'residual'
        where['3'] = 'mod9'
        return where

    def residuals(self) -> list[int]:
        return [int(q) for q, place in self.coverage().items() if place == 'residual']

    def filter_order(self) -> list[int]:
        """Residual filters in execution order: the strong ones (9 and the q = 1 mod 3, which
        keep about a third of the residues) ascending, then the rest ascending
        (pseudocube/gpu.py:134, pseudocube/batch_experiment.py:84-86)."""
        residuals = self.residuals()
        strong = sorted(q for q in residuals if q == 9 or q % 3 == 1)
        return strong + sorted(q for q in residuals if q != 9 and q % 3 != 1)

    def filter_groups(self) -> list[list[int]]:
        order = self.filter_order()
        return [order[k:k + 4] for k in range(0, len(order), 4)]

    def manifest(self) -> dict[str, Any]:
        af, bf = self.focuses()
        max_u = self._max_u()
        bounds = dict(max_u=str(max_u), max_v=str(self.B - 1), max_uB=str(max_u * self.B),
                      max_vA=str((self.B - 1) * self.A), x_bits=self.hi.bit_length(),
                      product_bits=(max_u * self.B).bit_length())
        return dict(schema_version=1, search_type='pseudocube', p=self.p, lo_exclusive=str(self.lo),
                    hi_inclusive=str(self.hi), A=str(self.A), B=str(self.B), canonical='v-in-[0,B)',
                    coverage=self.coverage(), table_sha256=definition(self.p)['sha256'],
                    focus_counts=[str(af.count), str(bf.count)], arithmetic_bounds=bounds)


@dataclass(frozen=True)
class Tile:
    """A canonical v range [first, end)."""
    first: int
    end: int

    def validate(self, config: Config) -> None:
        if not 0 <= self.first < self.end <= config.B:
            raise ValueError('tile must be a nonempty canonical v interval')

    def envelope(self, config: Config) -> dict[str, str]:
        """Inclusive u and v extremes of the tile and the conservative x extremes they imply."""
        self.validate(config)
        u_min, u_max = config.u_interval(self.first)[0], config.u_interval(self.end - 1)[1] - 1
        v_min, v_max = self.first, self.end - 1
        return dict(u_min=str(u_min), u_max=str(u_max), v_min=str(v_min), v_max=str(v_max),
                    x_min=str(u_min * config.B - v_max * config.A), x_max=str(u_max * config.B - v_min * config.A))

    def split(self) -> tuple['Tile', 'Tile']:
        """Halves at the integer middle: no overlap, no gap."""
        if self.end - self.first < 2:
            raise ValueError('unsplittable tile')
        middle = (self.first + self.end) // 2
        return Tile(self.first, middle), Tile(middle, self.end)

    def manifest(self, config: Config) -> dict[str, Any]:
        return dict(kind='v-window', first=str(self.first), end=str(self.end), envelope=self.envelope(config))


def targeted_coordinates(config: Config, n: int, radius: int = 1) -> tuple[list[int], list[int]]:
    """The CRT index neighbourhoods (radius on each side) of n's canonical pair in each focus; the
    matcher finds n from them, n itself is never injected."""
    u, v = config.canonical(n)
    af, bf = config.focuses()
    u_period, u_index = af.rank(u)
    v_period, v_index = bf.rank(v)
    if v_period != 0:
        raise ValueError('noncanonical v')
    near = lambda focus, index: (max(0, index - radius), min(focus.count, index + radius + 1))
    return (list(af.indices(*near(af, u_index), u_period)), list(bf.indices(*near(bf, v_index))))
