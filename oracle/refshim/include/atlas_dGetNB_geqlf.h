/* Stand-in for a generated tuned-NB header: no tuned block size, so ilaenv takes its default. */
