"""B200-native (sm_100a) doubly-focused pseudocube sieve.

Host modules mirror the reference's ``pseudocube`` call surface; the arithmetic runs in
``_lib/libpcube.so`` (CUDA sources in ``csrc/``, C ABI in ``include/pcube.h``).

    pseudocube.oracle            -> psuedocubes_b200.predicate
    pseudocube.tables / focus    -> psuedocubes_b200.tables / focus
    pseudocube.accounting        -> psuedocubes_b200.accounting (encoded, digest, durable)
    pseudocube.gpu               -> psuedocubes_b200.gpu
    pseudocube.batch_experiment  -> psuedocubes_b200.batch_experiment
    pseudocube.optimized         -> psuedocubes_b200.optimized
    pseudocube.multi.validate_result -> psuedocubes_b200.multi
    review/verify_cube.verify    -> psuedocubes_b200.verify
    tools/run_production.compute_batch -> psuedocubes_b200.run_production
    tools/reproduce.py           -> python -m psuedocubes_b200.reproduce
"""
__version__ = '0.1.0'
