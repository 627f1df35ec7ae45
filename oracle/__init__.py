"""CPU checkers for the CUDA propagator -- TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  The shipped library never does.

Two checkers live here:

* ``libtwi_oracle.so`` (``twi_oracle.cpp``): an own restatement of TorchWI's
  CPU propagator, templated on the storage type.  Its float build is pinned
  bit-for-bit to the reference and its double build is the FP64 run of the
  same scheme used to state each result's error.
* ``_ref/libtd2d_ref.so``: the reference's own CPU propagator compiled from
  its unmodified sources (``Makefile``).  Present where the reference sources
  were available at build time; the tests skip what needs it otherwise.
"""

from .oracle import (  # noqa: F401
    OracleError,
    build,
    have_ref,
    pad_model,
    ref_backward,
    ref_forward,
    ref_forward_only,
    twio_backward,
    twio_exa_backward,
    twio_exa_forward,
    twio_forward,
    shot_gather,
    shot_gradient,
)
