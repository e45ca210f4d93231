// The reference includes "PrivateDefs.h"; the file is privateDefs.h (case-insensitive on its platform).
#include "privateDefs.h"
