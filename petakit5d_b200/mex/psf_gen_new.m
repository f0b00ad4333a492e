function [ psf ] = psf_gen_new(psf, dz_psf, dz_data, medFactor, PSFGenMethod)
% Drop-in for microscopeDataProcessing/decon/psf_gen_new.m (GPU preparation through pkdecon_mex;
% same arguments, defaults and output; the output is single).
if nargin < 4
    medFactor = 1.5;
end
if nargin < 5
    PSFGenMethod = 'masked';
end
psf = pkdecon_mex('psf_gen', single(psf), dz_psf, dz_data, medFactor, lower(PSFGenMethod));
end
