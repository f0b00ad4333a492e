function [b_omw, OTF_bp_omw, abs_OTF_c, OTF_mask] = omw_backprojector_generation(psf, alpha, skewed, varargin)
% Drop-in for microscopeDataProcessing/decon/omw_backprojector_generation.m (GPU generation through
% pkdecon_mex; same parameters and outputs).
ip = inputParser;
ip.CaseSensitive = false;
ip.addRequired('psf');
ip.addRequired('alpha');
ip.addRequired('skewed');
ip.addParameter('OTFCumThresh', 0.9, @isnumeric);
ip.addParameter('OTFAreaThresh', 100, @isnumeric);
ip.addParameter('hannWinBounds', [0.8, 1], @(x) isnumeric(x) && numel(x) == 2);
ip.addParameter('minIntThrsh', 1e-3, @(x) isnumeric(x));
ip.parse(psf, alpha, skewed, varargin{:});
pr = ip.Results;
[b_omw, OTF_bp_omw, abs_OTF_c, mask] = pkdecon_mex('omw_bp', single(psf), alpha, skewed, pr.OTFCumThresh, ...
    pr.OTFAreaThresh, pr.hannWinBounds, pr.minIntThrsh);
OTF_mask = mask > 0;
end
