// Severity.h : TEST INFRASTRUCTURE ONLY — the severity enumeration of the plog logging library, as
// a minimal stand-in written for this repository (the reference's SEventConfig.hh names the type).
#pragma once
namespace plog {
enum Severity { none = 0, fatal = 1, error = 2, warning = 3, info = 4, debug = 5, verbose = 6 };
}
