/* Empty stand-in: the reference estimator includes this GSL header but links no GSL symbol. */
