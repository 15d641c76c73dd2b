/*
 * Link stubs for the oracle builds of the reference's known-answer models
 * (test infrastructure).  model/ldi2/model.c does not define two functions
 * of the model interface (src/model.h) that the core still references:
 * get_model_sigma (used by the kappa distribution and the trace output) and
 * get_model_beta (same).  Neither is reached by the custom-emission path the
 * ldi2 runs use; like the other test models (model/analytic/model.c:315-316)
 * they return 0.  Weak, so a model that defines them wins.
 */
double get_model_sigma(double X[4]) __attribute__((weak));
double get_model_beta(double X[4]) __attribute__((weak));
double get_model_sigma(double X[4]) { (void)X; return 0.; }
double get_model_beta(double X[4]) { (void)X; return 0.; }
