"""petakit5d_b200: B200 (sm_100a) Richardson-Lucy / OMW deconvolution behind a MATLAB-style C ABI.

Modules:
  decon          -- decon_lucy_function / decon_lucy_omw_function drop-ins (and device-pointer forms)
  backprojector  -- omw_backprojector_generation / BackProjector (every bp_type)
  chunking       -- findGoodFactorNumber, XR_zarrChunkCoordinatesExtraction, batched chunk decon,
                    RLdecon_large_in_memory / RLdecon_large_in_place (large-file runners)
  psfgen         -- psf_gen_new (PSF preparation) and RLdecon's PSF crops
  deskew         -- deskewRotateFrame3D (combined deskew / rotate after deconvolution)
  taper          -- edgetaper of every z slice and fspecial('gaussian') (RLdecon's nTapering)
  rldecon        -- RLdecon (per-file driver: files in, files out)
  tiff, zarrio   -- readtiff / writetiff / getImageSize, readzarr / writezarr
  serve          -- device-resident serving loop with continuous batching
  synth          -- seeded synthetic volumes and PSFs
"""
__version__ = "0.1.0"
