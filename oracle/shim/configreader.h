/* Oracle shim (test infrastructure only): Corsair ConfigReader placeholder.
 * The oracle driver sets Hybrid:: parameters directly, so no parsing occurs. */
#ifndef RHSHIM_CONFIGREADER_H
#define RHSHIM_CONFIGREADER_H
#include <string>
class ConfigReader { };
#endif
