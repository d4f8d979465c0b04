/* Stand-in for ITK's itkMacro.h, enough to compile RTK's CUDA back projector
 * and utilities (src/rtkCudaFDKBackProjectionImageFilter.cu,
 * src/rtkCudaUtilities.cu) without ITK: its exception macro and size type.
 * TEST INFRASTRUCTURE ONLY (timing and convention checks of the reference's
 * own CUDA kernel). */
#ifndef RTKB_STUB_ITKMACRO_H
#define RTKB_STUB_ITKMACRO_H
#include <sstream>
#include <stdexcept>
namespace itk
{
using SizeValueType = unsigned long;
}
#define itkGenericExceptionMacro(x)                                                                                    \
  {                                                                                                                    \
    std::ostringstream rtkb_message;                                                                                   \
    rtkb_message << "RTK CUDA error: " x;                                                                              \
    throw std::runtime_error(rtkb_message.str());                                                                      \
  }
#endif
