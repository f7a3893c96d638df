"""The reference's production ledger surface, re-exported unchanged: load_production,
save_compressed and Frontier (pseudocube/production.py:15-130 of the reference project).

The ledger is host-side durability code with no device work, so this library does not rebuild
it.  A worker commits this library's receipts (optimized.compute_lease, compute_leases) through
it exactly as through the reference's own; tests/test_ledger.py does so.  Importing this module
needs the reference's pseudocube package on the import path.
"""
from __future__ import annotations

try:
    from pseudocube.production import Frontier, load_production, save_compressed
except ImportError as exc:
    raise ImportError("psuedocubes_b200.production re-exports the reference project's pseudocube.production: "
                      "put the reference's pseudocube package on the import path") from exc

__all__ = ['Frontier', 'load_production', 'save_compressed']
