// Scene files: Wavefront OBJ + MTL, camera and area-light configurations.
//
// Host code.  The readers restate the reference's own parsers line by line
// in behaviour, so that a scene loads into the same vertices, faces,
// materials, camera and light as in the reference:
//  * FWObject::read + readMtlLib (src/Loaders/FWObjectReader.cpp:96-502);
//  * CameraManager::read (src/Loaders/CameraManager.cpp:94-158) and its
//    rotate (src/Loaders/CameraManager.cpp:29-63);
//  * LightSourceLoader::loadFromFile (src/Loaders/LightSourceLoader.cpp:26-89).
// Differences, each an error the reference would not detect: a face index
// that is not positive or that names a vertex past the end makes the whole
// file SHN_ERR_INVALID (the reference stores index - 1 and reads out of
// bounds later), and an .mtl file that cannot be opened is SHN_ERR_INVALID
// (the reference throws).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "internal.h"

struct shn_obj {
  struct Material {
    std::string name;
    float diffuse[3] = {0.f, 0.f, 0.f}, specular[3] = {0.f, 0.f, 0.f}, ambient[3] = {0.f, 0.f, 0.f};
    float spec_exp = 0.f;
  };
  struct Face {
    long long v[3], t[3], n[3];  // 0-based; -1 when absent
    uint32_t material;
  };
  std::vector<float> vertices;  // xyz triples
  std::vector<float> normals;
  std::vector<float> texcoords;
  std::vector<Face> faces;
  std::vector<Material> materials;
  std::string error;
  uint64_t skipped_lines = 0;  // lines the reference's parser rejects or does not know
};

namespace {

void skip_ws(const char*& s) {
  while (isspace((unsigned char)*s)) ++s;
}

std::string trim_end(const char* s) {
  size_t len = strlen(s);
  while (len > 0 && isspace((unsigned char)s[len - 1])) --len;
  return std::string(s, len);
}

std::string dir_of(const std::string& path) {
  const size_t k = path.find_last_of('/');
  if (k == std::string::npos) return ".";
  if (k == 0) return "/";
  return path.substr(0, k);
}

// One "v", "vn" or "vt" line after its keyword: floats read with strtod and
// narrowed to float, at most three of them; anything else on the line (a
// fourth value, a trailing comment) rejects the line, as in the reference.
bool parse_floats(const char* s, float out[3], int* count) {
  int k = 0;
  for (;;) {
    skip_ws(s);
    if (*s == 0) break;
    char* e = nullptr;
    const double d = strtod(s, &e);
    if (e == s) return false;
    s = e;
    if (k >= 3) return false;
    out[k++] = (float)d;
  }
  *count = k;
  return true;
}

// One "f" line after its keyword: vertex references v, v/t, v//n, v/t/n
// (1-based), with the reference's handling of the optional parts.  Returns
// false for a line the reference rejects; idx receives (v, t, n) triples as
// index - 1 (absent parts -1).
bool parse_face(const char* s, std::vector<long long>& idx) {
  constexpr size_t kMaxEntries = 4096 * 3;  // the reference's index buffer
  idx.clear();
  for (;;) {
    if (idx.size() + 3 >= kMaxEntries) return false;
    char* e = nullptr;
    long v = strtol(s, &e, 10);
    if (e == s) return false;
    s = e;
    idx.push_back((long long)v - 1);
    skip_ws(s);
    if (*s == '/') {
      ++s;
      skip_ws(s);
      if (*s != '/') {
        v = strtol(s, &e, 10);
        if (e == s) return false;
        s = e;
        idx.push_back((long long)v - 1);
      } else {
        idx.push_back(-1);
      }
      skip_ws(s);
      if (*s == '/') {
        ++s;
        skip_ws(s);
        v = strtol(s, &e, 10);
        // look one token ahead: the normal index counts only when what
        // follows it starts another vertex, or ends the line after a number
        const char* ahead = e;
        skip_ws(ahead);
        if (isdigit((unsigned char)*ahead) || ((*ahead == 0 || *ahead == '#') && s != e)) {
          if (s == e) return false;
          s = e;
          idx.push_back((long long)v - 1);
        } else {
          idx.push_back(-1);
        }
      } else {
        idx.push_back(-1);
      }
    } else {
      idx.push_back(-1);
      idx.push_back(-1);
    }
    skip_ws(s);
    if (*s == 0) break;
  }
  return idx.size() > 6;
}

// readMtlLib: Kd / Ks / Ka / Ns of the materials the OBJ file uses.  A
// "newmtl" naming a material the OBJ does not use is rejected and leaves the
// current material unchanged (so that its coefficients land on the previous
// material, as in the reference).
bool read_mtl(const std::string& path, shn_obj* o, const std::map<std::string, size_t>& index) {
  std::ifstream in(path.c_str(), std::ios::in | std::ios::binary);
  if (in.fail()) return false;
  std::string buf;
  long long cur = -1;
  while (std::getline(in, buf)) {
    const char* s = buf.c_str();
    skip_ws(s);
    if (strncasecmp(s, "newmtl", 6) == 0) {
      s += 6;
      skip_ws(s);
      const auto it = index.find(trim_end(s));
      if (it == index.end()) {
        ++o->skipped_lines;
        continue;
      }
      cur = (long long)it->second;
    } else if (strncasecmp(s, "Kd", 2) == 0 || strncasecmp(s, "Ks", 2) == 0 || strncasecmp(s, "Ka", 2) == 0) {
      const char kind = s[1];
      if (cur < 0) {
        ++o->skipped_lines;
        continue;
      }
      s += 2;
      float c[3];
      bool ok = true;
      for (int i = 0; i < 3 && ok; ++i) {
        skip_ws(s);
        char* e = nullptr;
        c[i] = (float)strtod(s, &e);
        if (e == s) ok = false;
        s = e;
      }
      if (!ok) {
        ++o->skipped_lines;
        continue;
      }
      shn_obj::Material& m = o->materials[(size_t)cur];
      float* dst = kind == 'd' ? m.diffuse : (kind == 'a' ? m.ambient : (kind == 's' ? m.specular : nullptr));
      if (dst) memcpy(dst, c, sizeof(c));
    } else if (strncasecmp(s, "Ns", 2) == 0) {
      if (cur < 0) {
        ++o->skipped_lines;
        continue;
      }
      s += 2;
      skip_ws(s);
      char* e = nullptr;
      const float v = (float)strtod(s, &e);
      if (e == s) {
        ++o->skipped_lines;
        continue;
      }
      o->materials[(size_t)cur].spec_exp = v;
    }
  }
  return true;
}

shn_status read_obj(const char* path, shn_obj* o) {
  std::ifstream in(path, std::ios::in);
  if (in.fail()) {
    o->error = std::string("cannot open ") + path;
    return SHN_ERR_INVALID;
  }
  shn_obj::Material def;
  def.name = "Default";
  for (int i = 0; i < 3; ++i) {
    def.diffuse[i] = .9774f;
    def.ambient[i] = 0.2f;
  }
  o->materials.push_back(def);
  std::map<std::string, size_t> index;
  index[def.name] = 0;
  std::vector<std::string> mtl_files;
  std::vector<long long> idx;
  uint32_t cur_mat = 0;
  std::string buf;
  while (std::getline(in, buf)) {
    const char* s = buf.c_str();
    skip_ws(s);
    const int c0 = tolower((unsigned char)*s);
    if (c0 == 0 || c0 == 'o' || c0 == 'g' || c0 == 's' || c0 == '#') continue;
    if (c0 == 'v') {
      ++s;
      int kind;
      const int c1 = tolower((unsigned char)*s);
      if (c1 == 'n') {
        kind = 1;
        ++s;
      } else if (c1 == 't') {
        kind = 2;
        ++s;
      } else if (isspace((unsigned char)*s)) {
        kind = 0;
      } else {
        ++o->skipped_lines;
        continue;
      }
      float f[3];
      int k = 0;
      if (!parse_floats(s, f, &k) || (kind != 2 && k != 3) || (kind == 2 && k < 2)) {
        ++o->skipped_lines;
        continue;
      }
      std::vector<float>& dst = kind == 0 ? o->vertices : (kind == 1 ? o->normals : o->texcoords);
      dst.insert(dst.end(), f, f + (kind == 2 ? 2 : 3));
      continue;
    }
    if (c0 == 'f') {
      ++s;
      if (tolower((unsigned char)*s) == 'o') ++s;
      skip_ws(s);
      if (!parse_face(s, idx)) {
        ++o->skipped_lines;
        continue;
      }
      // a polygon becomes a fan of triangles around its first vertex
      for (size_t q = 3; q + 3 < idx.size(); q += 3) {
        shn_obj::Face f;
        f.v[0] = idx[0]; f.t[0] = idx[1]; f.n[0] = idx[2];
        f.v[1] = idx[q]; f.t[1] = idx[q + 1]; f.n[1] = idx[q + 2];
        f.v[2] = idx[q + 3]; f.t[2] = idx[q + 4]; f.n[2] = idx[q + 5];
        f.material = cur_mat;
        o->faces.push_back(f);
      }
      continue;
    }
    if (strncasecmp(s, "usemtl", 6) == 0) {
      s += 6;
      skip_ws(s);
      const std::string name = trim_end(s);
      if (name.empty()) {
        ++o->skipped_lines;
        continue;
      }
      auto it = index.find(name);
      if (it == index.end()) {
        shn_obj::Material m;
        m.name = name;
        o->materials.push_back(m);
        it = index.emplace(name, o->materials.size() - 1).first;
      }
      cur_mat = (uint32_t)it->second;
      continue;
    }
    if (strncasecmp(s, "mtllib", 6) == 0) {
      s += 6;
      skip_ws(s);
      const std::string name = trim_end(s);
      if (name.empty()) {
        ++o->skipped_lines;
        continue;
      }
      mtl_files.push_back(name);
      continue;
    }
    ++o->skipped_lines;  // an entity the reference does not know
  }
  const std::string dir = dir_of(path);
  for (const std::string& f : mtl_files) {
    const std::string p = dir + "/" + f;
    if (!read_mtl(p, o, index)) {
      o->error = "cannot open " + p;
      return SHN_ERR_INVALID;
    }
  }
  // Material::setupPhongCoefficients (src/Loaders/FWObject.hpp:87-91)
  const float pi = (float)M_PI;
  for (shn_obj::Material& m : o->materials) {
    for (int i = 0; i < 3; ++i) {
      m.diffuse[i] = m.diffuse[i] / pi;
      m.specular[i] = ((m.specular[i] * (m.spec_exp + 2.f)) * 0.5f) / pi;
    }
  }
  const long long nv = (long long)(o->vertices.size() / 3);
  if (nv >= (1ll << 30) || o->faces.size() >= (1ull << 30)) {
    o->error = "more than 2^30 vertices or faces";
    return SHN_ERR_INVALID;
  }
  for (size_t i = 0; i < o->faces.size(); ++i)
    for (int k = 0; k < 3; ++k)
      if (o->faces[i].v[k] < 0 || o->faces[i].v[k] >= nv) {
        o->error = "face " + std::to_string(i) + " names a vertex outside the file";
        return SHN_ERR_INVALID;
      }
  return SHN_OK;
}

// A config line as CameraManager::read / LightSourceLoader::loadFromFile
// take it: lines holding a '#' anywhere are skipped whole; the first word
// names the entry; values are read by the stream (float parsing as strtof).
template <class F>
bool for_each_entry(const char* path, bool camera_eof_rule, F&& take) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  while (!in.eof()) {
    std::getline(in, line);
    while (line.find('#') != std::string::npos) {
      // the camera reader stops eating comment lines at the end of the file
      // and parses the last one; the light reader keeps reading
      if (camera_eof_rule && in.eof()) break;
      if (!camera_eof_rule && in.eof()) {
        line.clear();
        break;
      }
      std::getline(in, line);
    }
    std::stringstream ss(line);
    std::string key;
    ss >> key;
    take(key, ss);
  }
  return true;
}

void read3(std::stringstream& ss, float v[3]) { ss >> v[0] >> v[1] >> v[2]; }

void normalize3(float v[3]) {
  const float r = 1.0f / sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  v[0] = v[0] * r;
  v[1] = v[1] * r;
  v[2] = v[2] * r;
}

void cross3(const float a[3], const float b[3], float o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

}  // namespace

using namespace shn;

extern "C" {

shn_status shn_obj_read(const char* path, shn_obj** out) {
  if (!path || !out) return SHN_ERR_INVALID;
  *out = nullptr;
  shn_obj* o = new shn_obj();
  const shn_status rc = read_obj(path, o);
  if (rc != SHN_OK) {
    fprintf(stderr, "shn_obj_read: %s\n", o->error.c_str());
    delete o;
    return rc;
  }
  *out = o;
  return SHN_OK;
}

shn_status shn_obj_get_info(const shn_obj* o, shn_obj_info* info) {
  if (!o || !info) return SHN_ERR_INVALID;
  info->num_vertices = (uint32_t)(o->vertices.size() / 3);
  info->num_faces = (uint32_t)o->faces.size();
  info->num_materials = (uint32_t)o->materials.size();
  info->num_normals = (uint32_t)(o->normals.size() / 3);
  info->num_texcoords = (uint32_t)(o->texcoords.size() / 2);
  info->skipped_lines = o->skipped_lines;
  return SHN_OK;
}

shn_status shn_obj_copy(const shn_obj* o, float* vertices, uint32_t* faces, uint32_t* face_material,
                        float* diffuse, float* specular) {
  if (!o) return SHN_ERR_INVALID;
  if (vertices && !o->vertices.empty()) memcpy(vertices, o->vertices.data(), o->vertices.size() * sizeof(float));
  for (size_t i = 0; i < o->faces.size(); ++i) {
    if (faces)
      for (int k = 0; k < 3; ++k) faces[3 * i + k] = (uint32_t)o->faces[i].v[k];
    if (face_material) face_material[i] = o->faces[i].material;
  }
  for (size_t m = 0; m < o->materials.size(); ++m) {
    const shn_obj::Material& mt = o->materials[m];
    if (diffuse) {
      memcpy(diffuse + 4 * m, mt.diffuse, 12);
      diffuse[4 * m + 3] = 0.f;
    }
    if (specular) {
      memcpy(specular + 4 * m, mt.specular, 12);
      specular[4 * m + 3] = mt.spec_exp;
    }
  }
  return SHN_OK;
}

const char* shn_obj_material_name(const shn_obj* o, uint32_t m) {
  return (o && m < o->materials.size()) ? o->materials[m].name.c_str() : nullptr;
}

void shn_obj_destroy(shn_obj* o) { delete o; }

shn_status shn_camera_read(const char* path, shn_camera* cam) {
  if (!path || !cam) return SHN_ERR_INVALID;
  // entries missing from the file keep the values *cam holds on entry
  float pos[3], ori[3], up[3], rot[3] = {0.f, 0.f, 0.f};
  memcpy(pos, cam->eye, 12);
  memcpy(ori, cam->forward, 12);
  memcpy(up, cam->up, 12);
  float fov = cam->fov_deg;
  int rx = (int)cam->res_x, ry = (int)cam->res_y;
  const bool ok = for_each_entry(path, true, [&](const std::string& key, std::stringstream& ss) {
    if (key == "position") read3(ss, pos);
    else if (key == "orientation") read3(ss, ori);
    else if (key == "up") read3(ss, up);
    else if (key == "rotation") read3(ss, rot);
    else if (key == "resX") ss >> rx;
    else if (key == "resY") ss >> ry;
    else if (key == "FOV") ss >> fov;
  });
  if (!ok) return SHN_ERR_INVALID;
  // CameraManager::rotate: rotation about x, y, z (degrees) applied to the
  // orientation and the up vector
  const float pi = (float)M_PI;
  const float ax = rot[0] * pi / 180.f, ay = rot[1] * pi / 180.f, az = rot[2] * pi / 180.f;
  const float sx = sinf(ax), cx = cosf(ax), sy = sinf(ay), cy = cosf(ay), sz = sinf(az), cz = cosf(az);
  const float c1[3] = {cy * cz, sx * sy * cz - cx * sz, cx * sy * cz + sx * sz};
  const float c2[3] = {cy * sz, sx * sy * sz + cx * cz, sx * sy * sz - sx * cz};
  const float c3[3] = {-sy, sx * cy, cx * cy};
  float o2[3], u2[3];
  for (int i = 0; i < 3; ++i) {
    o2[i] = c1[i] * ori[0] + c2[i] * ori[1] + c3[i] * ori[2];
    u2[i] = c1[i] * up[0] + c2[i] * up[1] + c3[i] * up[2];
  }
  memcpy(cam->eye, pos, 12);
  memcpy(cam->forward, o2, 12);
  memcpy(cam->up, u2, 12);
  cam->fov_deg = fov;
  if (rx <= 0 || ry <= 0) return SHN_ERR_INVALID;
  cam->res_x = (uint32_t)rx;
  cam->res_y = (uint32_t)ry;
  return SHN_OK;
}

shn_status shn_light_read(const char* path, shn_area_light* l) {
  if (!path || !l) return SHN_ERR_INVALID;
  memset(l, 0, sizeof(*l));
  const bool ok = for_each_entry(path, false, [&](const std::string& key, std::stringstream& ss) {
    if (key == "position") read3(ss, l->position);
    else if (key == "normal") read3(ss, l->normal);
    else if (key == "intensity") read3(ss, l->intensity);
    else if (key == "edge1") read3(ss, l->edge1);
    else if (key == "edge2") read3(ss, l->edge2);
  });
  if (!ok) return SHN_ERR_INVALID;
  if (l->normal[0] == 0.f && l->normal[1] == 0.f && l->normal[2] == 0.f) {
    cross3(l->edge1, l->edge2, l->normal);
    normalize3(l->normal);
  }
  return SHN_OK;
}

}  // extern "C"
