function data = parallelReadTiff(filepath, range)
% Drop-in for the reference's parallelReadTiff MEX (io/cpp-tiff, called by io/readtiff.m):
% libpkdecon's multi-threaded TIFF reader (classic / BigTIFF, none / LZW / Deflate, ImageJ stacks).
if nargin < 2
    data = pkdecon_mex('readtiff', char(filepath));
else
    data = pkdecon_mex('readtiff', char(filepath), double(range));
end
end
