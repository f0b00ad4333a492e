function data = parallelReadZarr(filepath, varargin)
% Drop-in for the reference's parallelReadZarr MEX (io/cpp-zarr, called by io/readzarr.m) for arrays
% with none / zlib / gzip chunks: parallelReadZarr(filepath[, 'bbox', [y1 x1 z1 y2 x2 z2]]).
ip = inputParser;
ip.addParameter('bbox', [], @isnumeric);
ip.addParameter('sparse', true);
ip.parse(varargin{:});
data = pkdecon_mex('readzarr', char(filepath), double(ip.Results.bbox));
end
