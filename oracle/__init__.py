"""Test infrastructure only: the checkers the GPU path is compared against.

Nothing in the product (``ddfacet_b200``) imports this package.  It holds
  * ``ref``      -- a loader/driver for the reference's own CPU gridder/degridder
                    (DDFacet/Gridder, built from its sources by ``build_ref.sh`` into
                    ``oracle/_ref``), called with the reference's positional arguments;
  * ``fp64``     -- a plain-C FP64 restatement of the same gridder/degridder
                    (``gridder_fp64.c``, built by ``build_fp64.sh``), the "FP64 oracle";
  * ``dft``      -- FP64 numpy direct Fourier transforms (prediction and dirty image);
  * ``facets``   -- NumPy restatements of the per-facet transforms and stitching;
  * ``weights``  -- the imaging-weight pipeline restated.
"""
