function [pks, locs] = findpeaks(y)
% Local maxima of a vector with MATLAB's findpeaks semantics and no options, as
% pickFDC1.m calls it (core/pickFDC1.m:30, :40, :83, :93): a sample strictly
% larger than the sample before it and followed, after any run of equal
% samples, by a smaller one; a flat peak is reported at its first sample; the
% end points are never peaks.  Octave's signal package findpeaks differs, so
% put this directory on the Octave path only.
  v = y(:).';
  n = numel(v);
  locs = zeros(1, 0);
  k = 2;
  while k < n
    if v(k) > v(k - 1)
      j = k + 1;
      while j <= n && v(j) == v(k)
        j = j + 1;
      end
      if j <= n && v(j) < v(k)
        locs(end + 1) = k;
      end
      k = j;
    else
      k = k + 1;
    end
  end
  pks = v(locs);
  if iscolumn(y)
    pks = pks(:);
    locs = locs(:);
  end
end
