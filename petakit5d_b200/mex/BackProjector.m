function [PSF_bp, OTF_bp] = BackProjector(PSF_fp, bp_type, alpha, beta, n, resFlag, iRes, verboseFlag)
% Drop-in for third_parties/WBDeconvolution/BackProjector.m (GPU generation through pkdecon_mex;
% same bp_types, parameters, defaults and outputs; verboseFlag's printing and figure are not made).
if nargin < 2, bp_type = 'traditional'; end
if nargin < 3, alpha = 0.001; end
if nargin < 4, beta = 1; end
if nargin < 5, n = 10; end
if nargin < 6, resFlag = 1; end
if nargin < 7, iRes = [0, 0, 0]; end
[PSF_bp, OTF_bp] = pkdecon_mex('bp', single(PSF_fp), bp_type, alpha, beta, n, resFlag, iRes);
end
