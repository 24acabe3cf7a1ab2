function y = softmax(x)
% Column-wise softmax, shifted by each column's maximum, as the MATLAB Deep
% Learning Toolbox function that ADWDgrad_1.m calls (core/ADWDgrad_1.m:23, :57).
% Octave has no softmax; put this directory on the Octave path only.
  x = x - max(x, [], 1);
  e = exp(x);
  y = e ./ sum(e, 1);
end
