"""CPU oracles of zcmir's SMI path. Test infrastructure only: the tests, the smoke check and the
benchmark's CPU-baseline leg use them as the checker; the product never imports them."""
