function sz = getImageSizeMex(filepath)
% Drop-in for the reference's getImageSizeMex (io/cpp-tiff/mexSrc/getimagesizemex.cpp): [ny nx nz].
sz = pkdecon_mex('tiffsize', char(filepath));
end
