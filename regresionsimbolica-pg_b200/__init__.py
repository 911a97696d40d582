"""warpsymbolic_b200 -- B200-native evaluation and constant-fitting core for WarpSymbolic.

Drop-in for the reference's native extension `rpn_cuda_native` and its Python callers
(src/warpsymbolic/gpu/cuda_vm.py, evaluation.py).  The package directory is named
`regresionsimbolica-pg_b200`; it registers itself under the import name `warpsymbolic_b200`
(see __graft_entry__.load_package()).

  grammar      -- token vocabulary (mirror of gpu/grammar.py)
  cuda_vm      -- CudaRPNVM mirror (eval, eval_fused, eval_fitness)
  evaluation   -- GPUEvaluator mirror (evaluate_batch, validate_strict, ...)
  rpn_cuda_native -- the extension drop-in (same function names and signatures)
  population   -- GPUOperators' random generation and repair of invalid individuals
  reference_engine -- runs the reference's own estimator / engine on a chosen native module
  _native      -- ctypes binding of libwarpsym.so (include/warpsym.h)
"""
__version__ = "0.1.0"
