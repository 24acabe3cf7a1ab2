function parallel_init(ns)
% Octave stand-in for core/parallel_init.m: Octave has no gcp/parpool and runs
% parfor loops serially, so there is no pool to set up.  The batched engine
% (swd_engine_*) is the parallel path.
end
