"""B200-native two-component recursive-regularized D3Q27 TSLB step."""
