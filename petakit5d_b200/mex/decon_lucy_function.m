function [J_2, err_mat, k] = decon_lucy_function(I, PSF, NUMIT, varargin)
% Drop-in for microscopeDataProcessing/decon/decon_lucy_function.m (Biggs-accelerated RL): same
% signature and parameters (debug=true included); useGPU=false falls back to the original
% implementation, kept on the path as decon_lucy_function_matlab.m.
ip = inputParser;
ip.CaseSensitive = false;
ip.addRequired('I', @isnumeric);
ip.addRequired('PSF', @isnumeric);
ip.addRequired('NUMIT', @isnumeric);
ip.addParameter('Background', [], @isnumeric);
ip.addParameter('useGPU', true, @islogical);
ip.addParameter('save16bit', true, @islogical);
ip.addParameter('dampFactor', 1, @isnumeric);
ip.addParameter('scaleFactor', 1, @isnumeric);
ip.addParameter('deconOffset', 0, @isnumeric);
ip.addParameter('EdgeErosion', 0, @isnumeric);
ip.addParameter('bbox', [], @isnumeric);
ip.addParameter('debug', false, @islogical);
ip.addParameter('debug_folder', './debug/', @ischar);
ip.addParameter('saveStep', 1, @isnumeric);
ip.parse(I, PSF, NUMIT, varargin{:});
pr = ip.Results;
if ~pr.useGPU
    [J_2, err_mat, k] = decon_lucy_function_matlab(I, PSF, NUMIT, varargin{:});
    return;
end
opts = struct('Background', pr.Background, 'save16bit', pr.save16bit, 'dampFactor', pr.dampFactor, ...
    'scaleFactor', pr.scaleFactor, 'deconOffset', pr.deconOffset, 'EdgeErosion', pr.EdgeErosion, 'bbox', pr.bbox);
if pr.debug
    % err_mat and uint16(J_2) every saveStep iterations (decon_lucy_function.m:144-175)
    [J_2, err_mat, snaps] = pkdecon_mex('debug', 'rl', I, single(PSF), [], NUMIT, opts, pr.saveStep);
    mkdir(pr.debug_folder);
    for s = 1 : size(snaps, 4)
        writetiff(snaps(:, :, :, s), sprintf('%s/Iter_%04d.tif', pr.debug_folder, s * pr.saveStep));
    end
    k = NUMIT;
    return;
end
[J_2, k] = pkdecon_mex('rl', I, single(PSF), NUMIT, opts);
err_mat = zeros(NUMIT, 4);
end
