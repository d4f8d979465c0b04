// image_io.cpp -- MetaImage files (.mha with the data inline, .mhd with the
// data in a separate file), the format RTK's applications read and write
// through ITK's MetaImageIO (third-party: ITK's MetaIO library, not part of
// RTK; restated from its published header format).
//
// A header is "Key = Value" lines ending with ElementDataFile; the voxels
// follow in x-fastest order.  Keys used here: NDims (2 or 3), DimSize,
// ElementSpacing, Offset (physical position of the first voxel),
// TransformMatrix (the direction cosines of axis 0, then of axis 1, then of
// axis 2: the columns of ITK's direction matrix), ElementType (MET_FLOAT,
// MET_DOUBLE, MET_UCHAR, MET_CHAR, MET_USHORT, MET_SHORT, MET_UINT, MET_INT),
// BinaryDataByteOrderMSB, CompressedData (zlib), ElementNumberOfChannels (1)
// and ElementDataFile (LOCAL, or a file name relative to the header).
// MetaImage has no start index: a region with a non-zero index is written
// with Offset at the physical position of its first voxel, and read back with
// index 0.  Reading converts every element type to float32; writing stores
// float32.
#include "rtkb200.h"
#include "rtkb_internal.h"

#include <zlib.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace
{
using rtkb::fail;

struct Header
{
  int         ndims = 0;
  long long   dim[3] = { 1, 1, 1 };
  double      spacing[3] = { 1., 1., 1. };
  double      offset[3] = { 0., 0., 0. };
  double      tm[9] = { 1., 0., 0., 0., 1., 0., 0., 0., 1. }; // axis directions, one after the other
  std::string type = "MET_FLOAT";
  bool        msb = false;
  bool        compressed = false;
  int         channels = 1;
  std::string data_file = "LOCAL";
  size_t      data_start = 0; // byte offset of the data in the header's file (LOCAL)
};

std::string
trim(const std::string & s)
{
  size_t b = 0, e = s.size();
  while (b < e && std::isspace((unsigned char)s[b]))
    b++;
  while (e > b && std::isspace((unsigned char)s[e - 1]))
    e--;
  return s.substr(b, e - b);
}

bool
truthy(const std::string & v)
{
  const std::string t = trim(v);
  return t == "True" || t == "true" || t == "TRUE" || t == "1";
}

int
numbers(const std::string & v, double * out, int n, const std::string & key)
{
  std::istringstream iss(v);
  for (int i = 0; i < n; i++)
    if (!(iss >> out[i]))
      return fail(RTKB_ERR_INVALID_ARGUMENT, "MetaImage header: " + key + " needs " + std::to_string(n) + " numbers");
  return RTKB_OK;
}

int
read_header(const std::string & filename, std::ifstream & f, Header & h)
{
  std::string line;
  bool        end = false;
  while (!end && std::getline(f, line))
  {
    const size_t eq = line.find('=');
    if (eq == std::string::npos)
      continue;
    const std::string key = trim(line.substr(0, eq)), val = line.substr(eq + 1);
    int               rc = RTKB_OK;
    if (key == "NDims")
    {
      h.ndims = std::atoi(trim(val).c_str());
      if (h.ndims < 1 || h.ndims > 3)
        return fail(RTKB_ERR_UNSUPPORTED, "MetaImage: only 1-, 2- and 3-dimensional images are supported");
    }
    else if (key == "DimSize" || key == "ElementSpacing" || key == "Offset" || key == "Origin" || key == "Position")
    {
      if (h.ndims == 0)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "MetaImage header: " + key + " before NDims");
      double v[3];
      rc = numbers(val, v, h.ndims, key);
      for (int a = 0; a < h.ndims && rc == RTKB_OK; a++)
      {
        if (key == "DimSize")
          h.dim[a] = (long long)std::llround(v[a]);
        else if (key == "ElementSpacing")
          h.spacing[a] = v[a];
        else
          h.offset[a] = v[a];
      }
    }
    else if (key == "TransformMatrix" || key == "Rotation" || key == "Orientation")
    {
      if (h.ndims == 0)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "MetaImage header: " + key + " before NDims");
      double v[9];
      rc = numbers(val, v, h.ndims * h.ndims, key);
      for (int a = 0; a < h.ndims && rc == RTKB_OK; a++)
        for (int c = 0; c < h.ndims; c++)
          h.tm[3 * a + c] = v[h.ndims * a + c];
    }
    else if (key == "ElementType")
      h.type = trim(val);
    else if (key == "BinaryDataByteOrderMSB" || key == "ElementByteOrderMSB")
      h.msb = truthy(val);
    else if (key == "CompressedData")
      h.compressed = truthy(val);
    else if (key == "ElementNumberOfChannels")
      h.channels = std::atoi(trim(val).c_str());
    else if (key == "BinaryData" && !truthy(val))
      return fail(RTKB_ERR_UNSUPPORTED, "MetaImage: ASCII data is not supported");
    else if (key == "ElementDataFile")
    {
      h.data_file = trim(val);
      end = true;
    }
    if (rc != RTKB_OK)
      return rc;
  }
  if (!end)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "MetaImage header without ElementDataFile: " + filename);
  if (h.ndims == 0)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "MetaImage header without NDims: " + filename);
  if (h.channels != 1)
    return fail(RTKB_ERR_UNSUPPORTED, "MetaImage: only scalar images are supported");
  for (int a = 0; a < 3; a++)
    if (h.dim[a] <= 0 || h.dim[a] > 0x7fffffff)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "MetaImage: invalid DimSize");
  h.data_start = (size_t)f.tellg();
  return RTKB_OK;
}

int
element_size(const std::string & t)
{
  if (t == "MET_FLOAT" || t == "MET_INT" || t == "MET_UINT")
    return 4;
  if (t == "MET_DOUBLE")
    return 8;
  if (t == "MET_SHORT" || t == "MET_USHORT")
    return 2;
  if (t == "MET_CHAR" || t == "MET_UCHAR")
    return 1;
  return 0;
}

template <typename T>
float
load_elem(const unsigned char * p, bool swap)
{
  unsigned char b[sizeof(T)];
  for (size_t k = 0; k < sizeof(T); k++)
    b[k] = p[swap ? sizeof(T) - 1 - k : k];
  T v;
  std::memcpy(&v, b, sizeof(T));
  return (float)v;
}

void
convert(const std::string & t, const unsigned char * src, long long n, bool swap, float * dst)
{
  const int es = element_size(t);
  for (long long i = 0; i < n; i++)
  {
    const unsigned char * p = src + i * es;
    if (t == "MET_FLOAT")
      dst[i] = load_elem<float>(p, swap);
    else if (t == "MET_DOUBLE")
      dst[i] = load_elem<double>(p, swap);
    else if (t == "MET_INT")
      dst[i] = load_elem<int32_t>(p, swap);
    else if (t == "MET_UINT")
      dst[i] = load_elem<uint32_t>(p, swap);
    else if (t == "MET_SHORT")
      dst[i] = load_elem<int16_t>(p, swap);
    else if (t == "MET_USHORT")
      dst[i] = load_elem<uint16_t>(p, swap);
    else if (t == "MET_CHAR")
      dst[i] = load_elem<int8_t>(p, false);
    else
      dst[i] = load_elem<uint8_t>(p, false);
  }
}

bool
host_is_big_endian()
{
  const uint16_t one = 1;
  unsigned char  b;
  std::memcpy(&b, &one, 1);
  return b == 0;
}

std::string
directory_of(const std::string & path)
{
  const size_t s = path.find_last_of('/');
  return s == std::string::npos ? std::string() : path.substr(0, s + 1);
}

std::string
base_name(const std::string & path)
{
  const size_t s = path.find_last_of('/');
  return s == std::string::npos ? path : path.substr(s + 1);
}

bool
ends_with(const std::string & s, const char * suffix)
{
  const size_t n = std::strlen(suffix);
  return s.size() >= n && s.compare(s.size() - n, n, suffix) == 0;
}
} // namespace

extern "C" int
rtkb_image_read_mha(const char * filename, rtkb_image_desc * desc, float * data, long long capacity)
{
  if (!filename || !desc)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  try
  {
    std::ifstream f(filename, std::ios::binary);
    if (!f)
      return fail(RTKB_ERR_INVALID_ARGUMENT, std::string("cannot read image file ") + filename);
    Header h;
    int    rc = read_header(filename, f, h);
    if (rc != RTKB_OK)
      return rc;
    const int es = element_size(h.type);
    if (!es)
      return fail(RTKB_ERR_UNSUPPORTED, "MetaImage: unsupported ElementType " + h.type);
    rtkb_image_desc d{};
    for (int a = 0; a < 3; a++)
    {
      d.size[a] = (int)h.dim[a];
      d.index[a] = 0;
      d.origin[a] = h.offset[a];
      d.spacing[a] = h.spacing[a];
    }
    // TransformMatrix lists axis directions: row-major direction[r][c] = tm[c][r]
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++)
        d.direction[3 * r + c] = h.tm[3 * c + r];
    *desc = d;
    if (!data)
      return RTKB_OK;
    const long long n = h.dim[0] * h.dim[1] * h.dim[2];
    if (capacity < n)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "image buffer too small");
    std::vector<unsigned char> raw;
    {
      std::ifstream  df;
      std::ifstream * src = &f;
      if (h.data_file != "LOCAL")
      {
        if (h.data_file.find('%') != std::string::npos || h.data_file.rfind("LIST", 0) == 0)
          return fail(RTKB_ERR_UNSUPPORTED, "MetaImage: multi-file data is not supported");
        const std::string path = h.data_file[0] == '/' ? h.data_file : directory_of(filename) + h.data_file;
        df.open(path, std::ios::binary);
        if (!df)
          return fail(RTKB_ERR_INVALID_ARGUMENT, "cannot read MetaImage data file " + path);
        src = &df;
      }
      else
        f.seekg((std::streamoff)h.data_start);
      std::ostringstream ss;
      ss << src->rdbuf();
      const std::string bytes = ss.str();
      raw.assign(bytes.begin(), bytes.end());
    }
    const size_t need = (size_t)n * es;
    if (h.compressed)
    {
      std::vector<unsigned char> out(need);
      uLongf                     len = (uLongf)need;
      const int zr = uncompress(out.data(), &len, raw.data(), (uLong)raw.size());
      if (zr != Z_OK || len != need)
        return fail(RTKB_ERR_INVALID_ARGUMENT, std::string("MetaImage: corrupt compressed data in ") + filename);
      raw.swap(out);
    }
    if (raw.size() < need)
      return fail(RTKB_ERR_INVALID_ARGUMENT, std::string("MetaImage: data shorter than DimSize in ") + filename);
    convert(h.type, raw.data(), n, h.msb != host_is_big_endian(), data);
    return RTKB_OK;
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_image_write_mha(const char * filename, const rtkb_image_desc * desc, const float * data, int compress)
{
  std::string why;
  if (!filename || !desc || !data)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (!rtkb::desc_valid(desc, why))
    return fail(RTKB_ERR_INVALID_ARGUMENT, why);
  try
  {
    const std::string name(filename);
    const bool        detached = ends_with(name, ".mhd");
    if (!detached && !ends_with(name, ".mha"))
      return fail(RTKB_ERR_INVALID_ARGUMENT, "MetaImage file names end in .mha or .mhd");
    const long long n = (long long)desc->size[0] * desc->size[1] * desc->size[2];
    std::string     payload(reinterpret_cast<const char *>(data), (size_t)n * sizeof(float));
    if (compress)
    {
      uLongf                     len = compressBound((uLong)payload.size());
      std::vector<unsigned char> out(len);
      if (compress2(out.data(), &len, reinterpret_cast<const Bytef *>(payload.data()), (uLong)payload.size(),
                    Z_DEFAULT_COMPRESSION) != Z_OK)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "zlib compression failed");
      payload.assign(reinterpret_cast<const char *>(out.data()), len);
    }
    // Offset: the physical position of the region's first voxel
    double first[3];
    for (int r = 0; r < 3; r++)
    {
      first[r] = desc->origin[r];
      for (int c = 0; c < 3; c++)
        first[r] += desc->direction[3 * r + c] * desc->spacing[c] * desc->index[c];
    }
    std::ostringstream hdr;
    hdr << std::setprecision(17);
    hdr << "ObjectType = Image\nNDims = 3\nBinaryData = True\nBinaryDataByteOrderMSB = "
        << (host_is_big_endian() ? "True" : "False") << "\nCompressedData = " << (compress ? "True" : "False") << "\n";
    if (compress)
      hdr << "CompressedDataSize = " << payload.size() << "\n";
    hdr << "TransformMatrix =";
    for (int c = 0; c < 3; c++)
      for (int r = 0; r < 3; r++)
        hdr << ' ' << desc->direction[3 * r + c];
    hdr << "\nOffset = " << first[0] << ' ' << first[1] << ' ' << first[2] << "\nCenterOfRotation = 0 0 0"
        << "\nAnatomicalOrientation = RAI\nElementSpacing = " << desc->spacing[0] << ' ' << desc->spacing[1] << ' '
        << desc->spacing[2] << "\nDimSize = " << desc->size[0] << ' ' << desc->size[1] << ' ' << desc->size[2]
        << "\nElementType = MET_FLOAT\n";
    std::string data_name;
    if (detached)
    {
      data_name = base_name(name.substr(0, name.size() - 4)) + (compress ? ".zraw" : ".raw");
      hdr << "ElementDataFile = " << data_name << "\n";
    }
    else
      hdr << "ElementDataFile = LOCAL\n";
    std::ofstream f(name, std::ios::binary);
    if (!f)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "cannot write image file " + name);
    f << hdr.str();
    if (detached)
    {
      std::ofstream df(directory_of(name) + data_name, std::ios::binary);
      if (!df)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "cannot write image data file " + data_name);
      df.write(payload.data(), (std::streamsize)payload.size());
      if (!df)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "write failed: " + data_name);
    }
    else
      f.write(payload.data(), (std::streamsize)payload.size());
    return f ? RTKB_OK : fail(RTKB_ERR_INVALID_ARGUMENT, "write failed: " + name);
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}
