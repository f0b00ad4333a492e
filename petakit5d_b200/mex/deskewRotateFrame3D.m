function [volout] = deskewRotateFrame3D(vol, angle, dz, xyPixelSize, varargin)
% Drop-in for microscopeDataProcessing/deskew_rotate/deskewRotateFrame3D.m (GPU through pkdecon_mex;
% same parameters).  Linear interpolation without resampling runs on the GPU; cubic interpolation
% or a resampleFactor other than 1 raise pkdecon:unsupported (the reference's imwarp path).
ip = inputParser;
ip.CaseSensitive = false;
ip.addRequired('vol');
ip.addRequired('angle');
ip.addRequired('dz');
ip.addRequired('xyPixelSize');
ip.addParameter('reverse', false, @islogical);
ip.addParameter('Crop', true, @islogical);
ip.addParameter('bbox', [], @isnumeric);
ip.addParameter('objectiveScan', false, @islogical);
ip.addParameter('xStepThresh', 2.0, @isnumeric);
ip.addParameter('resampleFactor', [], @isnumeric);
ip.addParameter('gpuProcess', false, @islogical);
ip.addParameter('save16bit', false, @islogical);
ip.addParameter('interpMethod', 'linear', @(x) any(strcmpi(x, {'cubic', 'linear'})));
ip.parse(vol, angle, dz, xyPixelSize, varargin{:});
pr = ip.Results;
rs = pr.resampleFactor;
if ~strcmpi(pr.interpMethod, 'linear') || (~isempty(rs) && any(rs ~= 1))
    error('pkdecon:unsupported', 'cubic interpolation and resampling (the imwarp path) are not built');
end
if ~isa(vol, 'uint16')
    vol = single(vol);
end
volout = pkdecon_mex('dsr', vol, angle, dz, xyPixelSize, pr.reverse, pr.objectiveScan, pr.xStepThresh, ...
    double(pr.bbox), pr.save16bit);
end
