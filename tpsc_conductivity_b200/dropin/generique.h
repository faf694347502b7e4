// generique.h -- same header name as the reference's; the classes live in tpsc_dropin.h
#include "tpsc_dropin.h"
