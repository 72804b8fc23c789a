/* Empty stand-in: the oracle is a host-only build. */
