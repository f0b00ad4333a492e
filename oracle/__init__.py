"""CPU oracle for the Richardson-Lucy deconvolution hot path (TEST INFRASTRUCTURE ONLY).

This package restates, in numpy/scipy, the reference MATLAB functions of PetaKit5D's
deconvolution path so that the CUDA library can be checked against them:

* ``decon.py``         -- decon_psf2otf, decon_lucy_function (Biggs RL), decon_lucy_omw_function,
                          the pre/post-processing and decon_mask_edge_erosion.
* ``backprojector.py`` -- omw_backprojector_generation and the Wiener-Butterworth BackProjector.
* ``chunking.py``      -- findGoodFactorNumber and XR_zarrChunkCoordinatesExtraction.
* ``morph.py``         -- the binary morphology the OMW backprojector needs.
* ``psfgen.py``        -- psf_gen_new and the PSF crops of RLdecon.
* ``deskew.py``        -- deskewRotateFrame3D and its two MEX files.
* ``tiff.py``          -- TIFF / BigTIFF with TIFF LZW.
* ``zarrio.py``        -- Zarr v2 arrays (json, zlib, gzip).

Parity status: **unpinned**.  The reference is pure MATLAB (no MATLAB/Octave here) and ships no
test, golden vector or fixture for this path, so the restatement is pinned only by following the
cited lines, by analytic known answers (tests/test_oracle_kat.py) and by an FP64 variant.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may
import this package, and only as the checker.  The product (``petakit5d_b200``) never imports it.
"""
