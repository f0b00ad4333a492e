function parallelWriteTiff(filepath, data, mode, compression)
% Drop-in for the reference's parallelWriteTiff MEX (io/cpp-tiff, called by io/writetiff.m):
% BigTIFF, 512-row strips, LZW by default.  Only mode 'w' (write a new file) is supported.
if nargin >= 3 && ~isempty(mode) && ~strcmp(mode, 'w')
    error('pkdecon:unsupported', 'only mode ''w'' is supported');
end
if nargin < 4
    compression = 'lzw';
end
pkdecon_mex('writetiff', char(filepath), data, lower(compression));
end
