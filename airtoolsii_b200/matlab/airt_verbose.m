function airt_verbose(verbose, kmax, resnorms, relaxpars, timetaken)
%AIRT_VERBOSE  The iteration lines of the toolbox's verbose option, printed
%   after the GPU solve from the residual norms it returns (per-iteration
%   times are the mean over the solve).
k_final = numel(resnorms) - 1;
per = timetaken / max(k_final, 1);
for k = 1:k_final
    if verbose == 1 || (verbose > 1 && (k == 1 || k == k_final || mod(k, verbose) == 1))
        fprintf(['%*d/%d:  resnorm=%1.2e  relaxpar=%1.2e  ', ...
            'time(iter/total)=%1.2e/%1.2e secs.\n'], ceil(log10(kmax)), ...
            k, kmax, resnorms(k+1), relaxpars(min(k, numel(relaxpars))), per, per*k);
    end
end
end
