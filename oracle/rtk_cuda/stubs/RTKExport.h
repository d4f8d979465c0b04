/* Stand-in for RTK's CMake-generated RTKExport.h: symbol visibility macros
 * (every symbol of the test library is exported by default). */
#ifndef RTKB_STUB_RTKEXPORT_H
#define RTKB_STUB_RTKEXPORT_H
#define RTK_EXPORT
#endif
