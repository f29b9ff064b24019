/* Empty stand-in: the reference includes gsl_integration.h but never calls GSL. */
