function [J, err_mat] = decon_lucy_omw_function(I, PSF_f, PSF_b, NUMIT, varargin)
% Drop-in for microscopeDataProcessing/decon/decon_lucy_omw_function.m: same signature and
% name/value parameters; useGPU=true runs libpkdecon.so through pkdecon_mex (debug=true included),
% useGPU=false calls the original MATLAB implementation, kept on the path as
% decon_lucy_omw_function_matlab.m.
ip = inputParser;
ip.CaseSensitive = false;
ip.addRequired('I', @isnumeric);
ip.addRequired('PSF_f', @isnumeric);
ip.addRequired('PSF_b', @isnumeric);
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
ip.parse(I, PSF_f, PSF_b, NUMIT, varargin{:});
pr = ip.Results;
if ~pr.useGPU
    [J, err_mat] = decon_lucy_omw_function_matlab(I, PSF_f, PSF_b, NUMIT, varargin{:});
    return;
end
opts = struct('Background', pr.Background, 'save16bit', pr.save16bit, 'dampFactor', pr.dampFactor, ...
    'scaleFactor', pr.scaleFactor, 'deconOffset', pr.deconOffset, 'EdgeErosion', pr.EdgeErosion, 'bbox', pr.bbox);
if pr.debug
    % err_mat and uint16(J) every saveStep iterations (decon_lucy_omw_function.m:113-144)
    [J, err_mat, snaps] = pkdecon_mex('debug', 'omw', I, single(PSF_f), single(PSF_b), NUMIT, opts, pr.saveStep);
    mkdir(pr.debug_folder);
    for s = 1 : size(snaps, 4)
        writetiff(snaps(:, :, :, s), sprintf('%s/Iter_%04d.tif', pr.debug_folder, s * pr.saveStep));
    end
    return;
end
J = pkdecon_mex('omw', I, single(PSF_f), single(PSF_b), NUMIT, opts);
err_mat = zeros(NUMIT, 4);
end
