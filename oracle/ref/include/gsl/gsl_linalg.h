/* Forwards to the non-LTE stand-ins declared in gsl_vector.h (oracle harness only). */
#include "gsl_vector.h"
