// geometry_xml.cpp -- RTK's geometry file: rtk::ThreeDCircularProjectionGeometryXMLFileReader
// (src/rtkThreeDCircularProjectionGeometryXMLFileReader.cxx) and ...XMLFileWriter
// (src/rtkThreeDCircularProjectionGeometryXMLFileWriter.cxx), format documented in
// documentation/docs/Geometry.md:180-222.
//
// Reader: a <RTKThreeDCircularGeometry version="3"> document (version 2 is
// accepted as well).  Elements are matched case-insensitively by name;
// parameter elements outside <Projection> set values that every following
// projection inherits, those inside a <Projection> override them from there
// on; at </Projection> the projection is added (angles in degrees, "Angle" is
// an older name of "GantryAngle") with the current collimation, and the 3x4
// <Matrix> stored with it must agree with the one recomputed from the
// parameters to 0.001.  Writer: 15 significant digits; a parameter that is
// equal over all projections is written once before the projections (and
// not at all when it equals its default: 0, or unbounded for the
// collimation); the gantry angle and the matrix are written per projection.
#include "rtkb200.h"
#include "rtkb_internal.h"

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace
{
using rtkb::fail;

bool
iequal(const std::string & a, const char * b)
{
  size_t i = 0;
  for (; i < a.size() && b[i]; i++)
    if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i]))
      return false;
  return i == a.size() && !b[i];
}

std::string
decode_entities(const std::string & s)
{
  std::string out;
  out.reserve(s.size());
  for (size_t i = 0; i < s.size(); i++)
  {
    if (s[i] != '&')
    {
      out += s[i];
      continue;
    }
    static const std::pair<const char *, char> ents[] = { { "&lt;", '<' }, { "&gt;", '>' }, { "&amp;", '&' },
                                                          { "&quot;", '"' }, { "&apos;", '\'' } };
    bool done = false;
    for (const auto & e : ents)
    {
      const size_t n = std::char_traits<char>::length(e.first);
      if (s.compare(i, n, e.first) == 0)
      {
        out += e.second;
        i += n - 1;
        done = true;
        break;
      }
    }
    if (!done)
      out += '&';
  }
  return out;
}

struct Reader
{
  rtkb::Geometry & g;
  std::string      chars; // character data since the last start tag
  int              version = 0;
  bool             seen_root = false;
  double           ip = 0., oop = 0., ga = 0., sid = 0., sox = 0., soy = 0., sdd = 0., pox = 0., poy = 0.;
  double           cui = DBL_MAX, cus = DBL_MAX, cvi = DBL_MAX, cvs = DBL_MAX;
  double           mat[12] = {};
  bool             have_mat = false;

  int start(const std::string & name, const std::map<std::string, std::string> & atts)
  {
    chars.clear();
    if (name == "RTKThreeDCircularGeometry")
    {
      auto it = atts.find("version");
      version = it == atts.end() ? 0 : std::atoi(it->second.c_str());
      // version 3 reads version 2 files
      if (version != 3 && version != 2)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "Incompatible version of input geometry (v" + std::to_string(version) +
                                                 ") with current geometry (v3). You must re-generate your geometry "
                                                 "file again.");
      seen_root = true;
      g.p.clear();
    }
    if (iequal(name, "Projection"))
      have_mat = false;
    return RTKB_OK;
  }

  static int number(const std::string & s, double & v)
  {
    const char * b = s.c_str();
    char *       e = nullptr;
    v = std::strtod(b, &e);
    while (e && *e && std::isspace((unsigned char)*e))
      e++;
    if (e == b || (e && *e))
      return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: not a number: '" + s + "'");
    // an unbounded collimation (DBL_MAX) written with 15 digits reads back
    // just above DBL_MAX: keep it DBL_MAX rather than overflowing
    if (std::isinf(v))
      v = std::copysign(DBL_MAX, v);
    return RTKB_OK;
  }

  int end(const std::string & name)
  {
    struct Field
    {
      const char * tag;
      double *     dst;
    };
    const Field fields[] = { { "InPlaneAngle", &ip },
                             { "GantryAngle", &ga },
                             { "Angle", &ga },
                             { "OutOfPlaneAngle", &oop },
                             { "SourceToIsocenterDistance", &sid },
                             { "SourceOffsetX", &sox },
                             { "SourceOffsetY", &soy },
                             { "SourceToDetectorDistance", &sdd },
                             { "ProjectionOffsetX", &pox },
                             { "ProjectionOffsetY", &poy },
                             { "CollimationUInf", &cui },
                             { "CollimationUSup", &cus },
                             { "CollimationVInf", &cvi },
                             { "CollimationVSup", &cvs } };
    for (const Field & f : fields)
      if (iequal(name, f.tag))
        return number(chars, *f.dst);
    if (iequal(name, "RadiusCylindricalDetector"))
      return number(chars, g.radius_cylindrical);
    if (iequal(name, "Matrix"))
    {
      std::istringstream iss(chars);
      for (int k = 0; k < 12; k++)
        if (!(iss >> mat[k]))
          return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: a Matrix needs 12 numbers");
      have_mat = true;
      return RTKB_OK;
    }
    if (iequal(name, "Projection"))
    {
      const double d2r = std::atan(1.0) / 45.0;
      int rc = g.add_projection_rad(sid, sdd, d2r * ga, pox, poy, d2r * oop, d2r * ip, sox, soy);
      if (rc != RTKB_OK)
        return rc;
      auto & q = g.p.back();
      q.coll_uinf = cui;
      q.coll_usup = cus;
      q.coll_vinf = cvi;
      q.coll_vsup = cvs;
      if (have_mat)
        for (int k = 0; k < 12; k++)
          if (std::abs(mat[k] - q.mat[k]) > 0.001)
          {
            std::ostringstream m;
            m << "Matrix and parameters are not consistent (projection " << g.p.size() - 1 << ", entry " << k
              << ": file " << mat[k] << ", computed " << q.mat[k] << ")";
            return fail(RTKB_ERR_INVALID_ARGUMENT, m.str());
          }
    }
    return RTKB_OK;
  }
};

// A small XML pull parser: declarations, doctype and comments are skipped;
// elements with attributes, self-closing elements and character data (with
// the five predefined entities) are reported to the reader.
int
parse(const std::string & text, Reader & r)
{
  size_t i = 0;
  const size_t n = text.size();
  std::vector<std::string> open;
  while (i < n)
  {
    if (text[i] != '<')
    {
      const size_t j = text.find('<', i);
      r.chars += decode_entities(text.substr(i, (j == std::string::npos ? n : j) - i));
      i = (j == std::string::npos) ? n : j;
      continue;
    }
    if (text.compare(i, 4, "<!--") == 0)
    {
      const size_t j = text.find("-->", i + 4);
      if (j == std::string::npos)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: unterminated comment");
      i = j + 3;
      continue;
    }
    if (text.compare(i, 2, "<?") == 0 || text.compare(i, 2, "<!") == 0)
    {
      const size_t j = text.find('>', i);
      if (j == std::string::npos)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: unterminated declaration");
      i = j + 1;
      continue;
    }
    const size_t j = text.find('>', i);
    if (j == std::string::npos)
      return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: unterminated tag");
    std::string tag = text.substr(i + 1, j - i - 1);
    i = j + 1;
    if (!tag.empty() && tag[0] == '/')
    {
      std::string name = tag.substr(1);
      while (!name.empty() && std::isspace((unsigned char)name.back()))
        name.pop_back();
      if (open.empty() || open.back() != name)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: mismatched end tag </" + name + ">");
      open.pop_back();
      const int rc = r.end(name);
      if (rc != RTKB_OK)
        return rc;
      continue;
    }
    const bool self_closing = !tag.empty() && tag.back() == '/';
    if (self_closing)
      tag.pop_back();
    size_t k = 0;
    while (k < tag.size() && !std::isspace((unsigned char)tag[k]))
      k++;
    const std::string                  name = tag.substr(0, k);
    std::map<std::string, std::string> atts;
    while (k < tag.size())
    {
      while (k < tag.size() && std::isspace((unsigned char)tag[k]))
        k++;
      const size_t eq = tag.find('=', k);
      if (k >= tag.size() || eq == std::string::npos)
        break;
      std::string key = tag.substr(k, eq - k);
      while (!key.empty() && std::isspace((unsigned char)key.back()))
        key.pop_back();
      size_t q = eq + 1;
      while (q < tag.size() && std::isspace((unsigned char)tag[q]))
        q++;
      if (q >= tag.size() || (tag[q] != '"' && tag[q] != '\''))
        return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: unquoted attribute in <" + name + ">");
      const size_t qe = tag.find(tag[q], q + 1);
      if (qe == std::string::npos)
        return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: unterminated attribute in <" + name + ">");
      atts[key] = decode_entities(tag.substr(q + 1, qe - q - 1));
      k = qe + 1;
    }
    int rc = r.start(name, atts);
    if (rc != RTKB_OK)
      return rc;
    if (self_closing)
    {
      rc = r.end(name);
      if (rc != RTKB_OK)
        return rc;
    }
    else
      open.push_back(name);
  }
  if (!open.empty())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: unclosed element <" + open.back() + ">");
  if (!r.seen_root)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "geometry file: no RTKThreeDCircularGeometry element");
  return RTKB_OK;
}

// WriteLocalParameter: <name>value</name> at two indents, 15 significant digits
void
local_param(std::ostream & out, const std::string & indent, double v, const char * name)
{
  out << indent << indent << '<' << name << '>' << v << "</" << name << '>' << '\n';
}

// WriteGlobalParameter: true when v is equal over all projections (written
// once unless it is the default)
bool
global_param(std::ostream & out, const std::string & indent, const std::vector<double> & v, const char * name,
             bool degrees = false, double def = 0.)
{
  for (double x : v)
    if (x != v[0])
      return false;
  if (v[0] != def)
    local_param(out, indent, degrees ? v[0] * 45. / std::atan(1.) : v[0], name);
  return true;
}
} // namespace

extern "C" int
rtkb_geometry_read_xml(const char * filename, rtkb_geometry ** out)
{
  if (!filename || !out)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  try
  {
    std::ifstream f(filename, std::ios::binary);
    if (!f)
      return fail(RTKB_ERR_INVALID_ARGUMENT, std::string("cannot read geometry file ") + filename);
    std::ostringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    if (text.empty())
      return fail(RTKB_ERR_INVALID_ARGUMENT, std::string("empty geometry file ") + filename);
    rtkb_geometry * g = new rtkb_geometry();
    Reader          r{ g->g };
    const int       rc = parse(text, r);
    if (rc != RTKB_OK)
    {
      delete g;
      return rc;
    }
    *out = g;
    return RTKB_OK;
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

extern "C" int
rtkb_geometry_write_xml(const rtkb_geometry * g, const char * filename)
{
  if (!g || !filename)
    return fail(RTKB_ERR_INVALID_ARGUMENT, "null argument");
  if (g->g.p.empty())
    return fail(RTKB_ERR_INVALID_ARGUMENT, "Geometry object is empty, cannot write it");
  try
  {
    const auto &        P = g->g.p;
    const size_t        n = P.size();
    std::vector<double> ga, sid, sdd, sox, soy, pox, poy, ip, oop, cui, cus, cvi, cvs;
    g->g.gantry_angles(ga);
    for (const auto & q : P)
    {
      sid.push_back(q.sid);
      sdd.push_back(q.sdd);
      sox.push_back(q.sox);
      soy.push_back(q.soy);
      pox.push_back(q.pox);
      poy.push_back(q.poy);
      ip.push_back(q.ip);
      oop.push_back(q.oop);
      cui.push_back(q.coll_uinf);
      cus.push_back(q.coll_usup);
      cvi.push_back(q.coll_vinf);
      cvs.push_back(q.coll_vsup);
    }
    std::ostringstream out;
    out.precision(15);
    const std::string indent("  ");
    out << "<?xml version=\"1.0\"?>\n<!DOCTYPE RTKGEOMETRY>\n<RTKThreeDCircularGeometry version=\"3\">\n";
    const bool gsid = global_param(out, indent, sid, "SourceToIsocenterDistance");
    const bool gsdd = global_param(out, indent, sdd, "SourceToDetectorDistance");
    const bool gsox = global_param(out, indent, sox, "SourceOffsetX");
    const bool gsoy = global_param(out, indent, soy, "SourceOffsetY");
    const bool gpox = global_param(out, indent, pox, "ProjectionOffsetX");
    const bool gpoy = global_param(out, indent, poy, "ProjectionOffsetY");
    const bool gip = global_param(out, indent, ip, "InPlaneAngle", true);
    const bool goop = global_param(out, indent, oop, "OutOfPlaneAngle", true);
    const bool gcui = global_param(out, indent, cui, "CollimationUInf", false, DBL_MAX);
    const bool gcus = global_param(out, indent, cus, "CollimationUSup", false, DBL_MAX);
    const bool gcvi = global_param(out, indent, cvi, "CollimationVInf", false, DBL_MAX);
    const bool gcvs = global_param(out, indent, cvs, "CollimationVSup", false, DBL_MAX);
    if (g->g.radius_cylindrical != 0.)
      local_param(out, indent, g->g.radius_cylindrical, "RadiusCylindricalDetector");
    const double r2d = 45. / std::atan(1.);
    for (size_t i = 0; i < n; i++)
    {
      out << indent << "<Projection>\n";
      local_param(out, indent, r2d * ga[i], "GantryAngle");
      if (!gsid)
        local_param(out, indent, sid[i], "SourceToIsocenterDistance");
      if (!gsdd)
        local_param(out, indent, sdd[i], "SourceToDetectorDistance");
      if (!gsox)
        local_param(out, indent, sox[i], "SourceOffsetX");
      if (!gsoy)
        local_param(out, indent, soy[i], "SourceOffsetY");
      if (!gpox)
        local_param(out, indent, pox[i], "ProjectionOffsetX");
      if (!gpoy)
        local_param(out, indent, poy[i], "ProjectionOffsetY");
      if (!gip)
        local_param(out, indent, r2d * ip[i], "InPlaneAngle");
      if (!goop)
        local_param(out, indent, r2d * oop[i], "OutOfPlaneAngle");
      if (!gcui)
        local_param(out, indent, cui[i], "CollimationUInf");
      if (!gcus)
        local_param(out, indent, cus[i], "CollimationUSup");
      if (!gcvi)
        local_param(out, indent, cvi[i], "CollimationVInf");
      if (!gcvs)
        local_param(out, indent, cvs[i], "CollimationVSup");
      out << indent << indent << "<Matrix>\n";
      for (int r = 0; r < 3; r++)
      {
        out << indent << indent << indent;
        for (int c = 0; c < 4; c++)
          out << std::setw(19) << P[i].mat[4 * r + c] << (c < 3 ? " " : "\n");
      }
      out << indent << indent << "</Matrix>\n" << indent << "</Projection>\n";
    }
    out << "</RTKThreeDCircularGeometry>\n";
    std::ofstream f(filename, std::ios::binary);
    if (!f)
      return fail(RTKB_ERR_INVALID_ARGUMENT, std::string("cannot write geometry file ") + filename);
    f << out.str();
    return f ? RTKB_OK : fail(RTKB_ERR_INVALID_ARGUMENT, std::string("write failed: ") + filename);
  }
  catch (...)
  {
    return fail(RTKB_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}
