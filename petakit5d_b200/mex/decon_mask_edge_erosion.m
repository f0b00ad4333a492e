function [mask] = decon_mask_edge_erosion(mask, EdgeErosion)
% Drop-in for microscopeDataProcessing/decon/decon_mask_edge_erosion.m (GPU erosion through pkdecon_mex;
% same arguments and logical output).
mask = pkdecon_mex('mask_erosion', uint16(mask > 0), EdgeErosion);
end
