// Object model and commit logic of the cuda device.
//
// Volume commit restates the reference's parameter handling and validation
// (openvkl/devices/cpu/volume/vdb/DenseVdbVolume.cpp:21-199,
// VdbVolume.cpp:398-1062) and builds the device-resident grid: the dense
// tree is generated on the GPU in closed form, the sparse tree is inserted on
// the host (first-come node numbering, as VdbVolume.cpp:244-331) and
// uploaded, and all value ranges are computed on the GPU (k_build.cu).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <unordered_set>

#include "kernels.h"
#include "objects.h"

namespace vklcuda {

size_t sizeOfType(VKLDataType t)
{
  switch (t) {
  case VKL_CHAR:
  case VKL_UCHAR:
    return 1;
  case VKL_SHORT:
  case VKL_USHORT:
  case VKL_HALF:
    return 2;
  case VKL_BOOL:
  case VKL_INT:
  case VKL_UINT:
  case VKL_FLOAT:
    return 4;
  case VKL_VEC2I:
  case VKL_VEC2UI:
  case VKL_VEC2F:
  case VKL_BOX1I:
  case VKL_BOX1F:
  case VKL_LONG:
  case VKL_ULONG:
  case VKL_DOUBLE:
  case VKL_VOID_PTR:
    return 8;
  case VKL_VEC3I:
  case VKL_VEC3UI:
  case VKL_VEC3F:
    return 12;
  case VKL_VEC4I:
  case VKL_VEC4UI:
  case VKL_VEC4F:
    return 16;
  case VKL_BOX2I:
  case VKL_BOX2F:
    return 16;
  case VKL_BOX3I:
  case VKL_BOX3F:
    return 24;
  case VKL_BOX4I:
  case VKL_BOX4F:
    return 32;
  case VKL_LINEAR3F:
    return 36;
  case VKL_AFFINE3F:
    return 48;
  default:
    if (t & VKL_OBJECT)
      return sizeof(VKLObject);
    return 0;
  }
}

// ---------------------------------------------------------------------------
// ManagedObject.
// ---------------------------------------------------------------------------
ManagedObject::~ManagedObject()
{
  for (auto &kv : params)
    if (kv.second.obj)
      kv.second.obj->refDec();
  if (heldDevice)
    heldDevice->refDec();
}

void Device::refDec()
{
  if (refs.fetch_sub(1) == 1)
    delete this;
}

void ManagedObject::setParam(const char *name, VKLDataType type, const void *mem)
{
  if (!name)
    fail("parameter name is NULL");
  Param p;
  p.type = type;
  if (type == VKL_STRING) {
    p.str = mem ? (const char *)mem : "";
  } else if (type & VKL_OBJECT) {
    const VKLObject *o = (const VKLObject *)mem;
    p.obj              = o ? (ManagedObject *)o->host : nullptr;
    if (p.obj)
      p.obj->refInc();
  } else {
    const size_t n = sizeOfType(type);
    if (!n)
      fail(std::string("unsupported parameter type for '") + name + "'");
    p.bytes.assign((const uint8_t *)mem, (const uint8_t *)mem + n);
  }
  auto it = params.find(name);
  if (it != params.end() && it->second.obj)
    it->second.obj->refDec();
  params[name] = std::move(p);
}

int ManagedObject::getInt(const std::string &name, int def) const
{
  const Param *p = find(name);
  if (!p)
    return def;
  if (p->type == VKL_INT || p->type == VKL_UINT || p->type == VKL_BOOL) {
    int v;
    std::memcpy(&v, p->bytes.data(), 4);
    return v;
  }
  if (p->type == VKL_FLOAT) {
    float f;
    std::memcpy(&f, p->bytes.data(), 4);
    return (int)f;
  }
  return def;
}

float ManagedObject::getFloat(const std::string &name, float def) const
{
  const Param *p = find(name);
  if (!p)
    return def;
  if (p->type == VKL_FLOAT) {
    float f;
    std::memcpy(&f, p->bytes.data(), 4);
    return f;
  }
  if (p->type == VKL_INT || p->type == VKL_UINT) {
    int v;
    std::memcpy(&v, p->bytes.data(), 4);
    return (float)v;
  }
  return def;
}

bool ManagedObject::getBool(const std::string &name, bool def) const
{
  const Param *p = find(name);
  if (!p || p->bytes.size() < 4)
    return def;
  int v;
  std::memcpy(&v, p->bytes.data(), 4);
  return v != 0;
}

void ManagedObject::getVec3f(const std::string &name, float out[3], const float def[3]) const
{
  const Param *p = find(name);
  if (p && p->type == VKL_VEC3F) {
    std::memcpy(out, p->bytes.data(), 12);
    return;
  }
  std::memcpy(out, def, 12);
}

void ManagedObject::getVec3i(const std::string &name, int out[3], const int def[3]) const
{
  const Param *p = find(name);
  if (p && (p->type == VKL_VEC3I || p->type == VKL_VEC3UI)) {
    std::memcpy(out, p->bytes.data(), 12);
    return;
  }
  std::memcpy(out, def, 12);
}

Data *ManagedObject::getData(const std::string &name) const
{
  const Param *p = find(name);
  if (!p || !p->obj)
    return nullptr;
  return dynamic_cast<Data *>(p->obj);
}

// ---------------------------------------------------------------------------
// Device.
// ---------------------------------------------------------------------------
void Device::ensurePipeline()
{
  if (copyIn)
    return;
  cudaCheck(cudaStreamCreateWithFlags(&copyIn, cudaStreamNonBlocking), "copy stream");
  cudaCheck(cudaStreamCreateWithFlags(&copyOut, cudaStreamNonBlocking), "copy stream");
  cudaCheck(cudaEventCreateWithFlags(&pipeStart, cudaEventDisableTiming), "copy event");
  for (int s = 0; s < kPipeSlots; ++s) {
    cudaCheck(cudaEventCreateWithFlags(&inReady[s], cudaEventDisableTiming), "copy event");
    cudaCheck(cudaEventCreateWithFlags(&computed[s], cudaEventDisableTiming), "copy event");
    cudaCheck(cudaEventCreateWithFlags(&drained[s], cudaEventDisableTiming), "copy event");
  }
}

Device::~Device()
{
  if (!copyIn)
    return;
  cudaStreamSynchronize(copyIn);
  cudaStreamSynchronize(copyOut);
  for (int s = 0; s < kPipeSlots; ++s) {
    cudaEventDestroy(inReady[s]);
    cudaEventDestroy(computed[s]);
    cudaEventDestroy(drained[s]);
  }
  cudaEventDestroy(pipeStart);
  cudaStreamDestroy(copyIn);
  cudaStreamDestroy(copyOut);
}

void Device::setError(VKLError code, const std::string &msg)
{
  lastErrorCode = code;
  lastErrorMsg  = msg;
  if (errorCb)
    errorCb(errorUser, code, msg.c_str());
}

void Device::log(int level, const std::string &msg)
{
  if (logCb && level >= logLevel)
    logCb(logUser, msg.c_str());
}

// ---------------------------------------------------------------------------
// Data.
// ---------------------------------------------------------------------------
Data::~Data()
{
  for (ManagedObject *o : objects)
    if (o)
      o->refDec();
}

const uint8_t *Data::hostBytes()
{
  if (host.empty() && numItems && dev) {
    host.resize(numItems * itemSize);
    cudaCheck(cudaMemcpy(host.data(), dev, host.size(), cudaMemcpyDeviceToHost), "Data readback");
  }
  return host.data();
}

// ---------------------------------------------------------------------------
// Volume commit.
// ---------------------------------------------------------------------------
namespace {

// Device memory a sparse volume may spend on its flat leaf map.
constexpr uint64_t kLeafMapBudgetBytes = 4ull << 30;

bool isVoxelType(VKLDataType t)
{
  return t == VKL_UCHAR || t == VKL_SHORT || t == VKL_USHORT || t == VKL_HALF ||
         t == VKL_FLOAT || t == VKL_DOUBLE;
}

// "indexToObject" as an affine3f parameter or a data array of >= 12 floats,
// column-major [vx vy vz p] (VdbVolume.h:37-57).
bool readIndexToObject(const ManagedObject &o, float c[12])
{
  const ManagedObject::Param *p = o.find("indexToObject");
  if (!p)
    return false;
  if (p->type == VKL_AFFINE3F) {
    std::memcpy(c, p->bytes.data(), 48);
    return true;
  }
  Data *d = o.getData("indexToObject");
  if (d && d->type == VKL_FLOAT && d->numItems >= 12) {
    std::memcpy(c, d->hostBytes(), 48);
    return true;
  }
  return false;
}

// Row-major 3x4 index->object and its inverse, inverted in FP64 and rounded
// once to FP32.
void makeTransforms(const float c[12], float *i2o, float *o2i)
{
  const double L[3][3] = {{c[0], c[3], c[6]}, {c[1], c[4], c[7]}, {c[2], c[5], c[8]}};
  const double p[3]    = {c[9], c[10], c[11]};
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k)
      i2o[r * 3 + k] = (float)L[r][k];
  i2o[9]  = c[9];
  i2o[10] = c[10];
  i2o[11] = c[11];
  const double det = L[0][0] * (L[1][1] * L[2][2] - L[1][2] * L[2][1]) -
                     L[0][1] * (L[1][0] * L[2][2] - L[1][2] * L[2][0]) +
                     L[0][2] * (L[1][0] * L[2][1] - L[1][1] * L[2][0]);
  if (det == 0.0)
    fail("indexToObject transform is singular");
  double I[3][3];
  I[0][0] = (L[1][1] * L[2][2] - L[1][2] * L[2][1]) / det;
  I[0][1] = (L[0][2] * L[2][1] - L[0][1] * L[2][2]) / det;
  I[0][2] = (L[0][1] * L[1][2] - L[0][2] * L[1][1]) / det;
  I[1][0] = (L[1][2] * L[2][0] - L[1][0] * L[2][2]) / det;
  I[1][1] = (L[0][0] * L[2][2] - L[0][2] * L[2][0]) / det;
  I[1][2] = (L[0][2] * L[1][0] - L[0][0] * L[1][2]) / det;
  I[2][0] = (L[1][0] * L[2][1] - L[1][1] * L[2][0]) / det;
  I[2][1] = (L[0][1] * L[2][0] - L[0][0] * L[2][1]) / det;
  I[2][2] = (L[0][0] * L[1][1] - L[0][1] * L[1][0]) / det;
  for (int r = 0; r < 3; ++r) {
    for (int k = 0; k < 3; ++k)
      o2i[r * 3 + k] = (float)I[r][k];
    o2i[9 + r] = (float)(-(I[r][0] * p[0] + I[r][1] * p[1] + I[r][2] * p[2]));
  }
}

// Attribute arrays from a "data"-like parameter: a single Data or a Data of
// Data (one per attribute).
std::vector<Data *> attributeArrays(const ManagedObject &o, const char *name)
{
  std::vector<Data *> out;
  Data *d = o.getData(name);
  if (!d)
    return out;
  if (d->type == VKL_DATA) {
    for (ManagedObject *m : d->objects) {
      Data *a = dynamic_cast<Data *>(m);
      if (!a)
        fail(std::string("'") + name + "' holds a non-data object");
      out.push_back(a);
    }
  } else {
    out.push_back(d);
  }
  return out;
}

float undefinedBackground()
{
  uint32_t bits = 0xFFC068B5u;
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

uint64_t packKey(uint32_t x, uint32_t y, uint32_t z)
{
  return ((uint64_t)x << 42) ^ ((uint64_t)y << 21) ^ (uint64_t)z;
}

}  // namespace

void TextureAtlas::release()
{
  if (tex)
    cudaDestroyTextureObject(tex);
  if (surf)
    cudaDestroySurfaceObject(surf);
  if (array)
    cudaFreeArray(array);
  tex = surf = 0;
  array = nullptr;
  width = height = 0;
}

bool TextureAtlas::ensure(uint32_t w, uint32_t h)
{
  if (array && w == width && h == height)
    return true;
  release();
  cudaChannelFormatDesc fmt = cudaCreateChannelDesc<float>();
  if (cudaMallocArray(&array, &fmt, w, h, cudaArraySurfaceLoadStore) != cudaSuccess) {
    cudaGetLastError();  // an atlas that does not fit is skipped, not an error
    array = nullptr;
    return false;
  }
  cudaResourceDesc res{};
  res.resType         = cudaResourceTypeArray;
  res.res.array.array = array;
  cudaTextureDesc td{};
  td.addressMode[0] = td.addressMode[1] = cudaAddressModeBorder;
  td.filterMode       = cudaFilterModePoint;
  td.readMode         = cudaReadModeElementType;
  td.normalizedCoords = 0;
  cudaCheck(cudaCreateSurfaceObject(&surf, &res), "atlas surface");
  cudaCheck(cudaCreateTextureObject(&tex, &res, &td, nullptr), "atlas texture");
  width  = w;
  height = h;
  return true;
}

std::unique_ptr<TextureAtlas> Device::takeAtlas(uint32_t width, uint32_t height)
{
  std::lock_guard<std::mutex> lock(atlasMutex);
  for (auto it = atlasPool.begin(); it != atlasPool.end(); ++it)
    if ((*it)->width == width && (*it)->height == height) {
      std::unique_ptr<TextureAtlas> a = std::move(*it);
      atlasPool.erase(it);
      return a;
    }
  return nullptr;
}

void Device::giveAtlas(std::unique_ptr<TextureAtlas> atlas)
{
  if (!atlas || !atlas->array)
    return;
  std::lock_guard<std::mutex> lock(atlasMutex);
  atlasPool.push_back(std::move(atlas));
  while (atlasPool.size() > kAtlasPool)
    atlasPool.erase(atlasPool.begin());
}

void Device::dropAtlases()
{
  std::lock_guard<std::mutex> lock(atlasMutex);
  atlasPool.clear();
}

Volume::~Volume()
{
  for (auto &a : atlases)
    if (a && device)
      device->giveAtlas(std::move(a));
}

namespace {

// Planes per atlas row for X x Y x Z float planes within the device's 2D
// texture and surface limits; 0 when the volume does not fit one atlas.
// Up to 64 planes side by side keep z-neighbours a few KB apart.  The count
// is a power of two, so the sampling kernels find a plane's tile with a
// shift and a mask instead of an integer division.
uint32_t atlasPlanesPerRow(int cudaDevice, uint32_t X, uint32_t Y, uint32_t Z)
{
  int tw = 0, th = 0, sw = 0, sh = 0;
  cudaDeviceGetAttribute(&tw, cudaDevAttrMaxTexture2DWidth, cudaDevice);
  cudaDeviceGetAttribute(&th, cudaDevAttrMaxTexture2DHeight, cudaDevice);
  cudaDeviceGetAttribute(&sw, cudaDevAttrMaxSurface2DWidth, cudaDevice);
  cudaDeviceGetAttribute(&sh, cudaDevAttrMaxSurface2DHeight, cudaDevice);
  const uint64_t maxW = (uint64_t)std::min(tw, sw), maxH = (uint64_t)std::min(th, sh);
  if (X == 0 || Y == 0 || Z == 0 || X > maxW)
    return 0;
  // the widest power of two up to 64 planes that fits the width and Z
  uint64_t T = 64;
  while (T > 1 && (T > Z || T * X > maxW))
    T >>= 1;
  // more planes per row when the rows would exceed the height
  while ((Z + T - 1) / T * Y > maxH) {
    T <<= 1;
    if (T * X > maxW)
      return 0;
  }
  return (uint32_t)T;
}

}  // namespace

void Volume::commit()
{
  // Work that still reads the previous commit's buffers (on any stream)
  // ends before they are reused, as it would before cudaFree.
  if (!buffers.empty())
    cudaCheck(cudaDeviceSynchronize(), "re-commit");
  recycled = std::move(buffers);
  buffers.clear();
  struct DropRecycled {
    Volume *v;
    ~DropRecycled() { v->recycled.clear(); }
  } dropRecycled{this};
  keep.clear();
  committed = false;
  grid      = DevGrid{};
  for (auto &m : macroRanges)
    m.reset();
  filter = getInt("filter", VKL_FILTER_LINEAR);
  gradientFilter = getInt("gradientFilter", filter);
  maxSamplingDepth = (uint32_t)std::min(getInt("maxSamplingDepth", (int)kNumLevels - 1),
                                        (int)kNumLevels - 1);
  // Temporal parameters describing temporally constant data are accepted,
  // as the reference accepts them: a structuredRegular volume is temporally
  // varying only with temporallyStructuredNumTimesteps > 0 or a
  // temporallyUnstructuredIndices array (DenseVdbVolume.cpp:149-186), a vdb
  // node only with a non-constant node.temporalFormat (checked in
  // commitVdb).  The reference's VdbVolumeBuffers utility sets the node.*
  // temporal arrays on every volume it creates.
  if (isDense)
    commitDense();
  else
    commitVdb();
  committed = true;
}

void Volume::finishCommit(const float lo[3], const float hi[3])
{
  // Domain box (VdbVolume.cpp:808-811) and object bounds (:814-824).
  for (int a = 0; a < 3; ++a) {
    grid.domain[a]     = lo[a] - (float)grid.rootOrigin[a];
    grid.domain[3 + a] = hi[a] - (float)grid.rootOrigin[a];
  }
  const float inf = INFINITY;
  float b[6]      = {inf, inf, inf, -inf, -inf, -inf};
  for (int i = 0; i < 8; ++i) {
    const float v[3] = {(i & 1) ? hi[0] : lo[0], (i & 2) ? hi[1] : lo[1], (i & 4) ? hi[2] : lo[2]};
    const float *M   = grid.indexToObject;
    const float w[3] = {M[0] * v[0] + M[1] * v[1] + M[2] * v[2] + M[9],
                        M[3] * v[0] + M[4] * v[1] + M[5] * v[2] + M[10],
                        M[6] * v[0] + M[7] * v[1] + M[8] * v[2] + M[11]};
    for (int a = 0; a < 3; ++a) {
      b[a]     = std::min(b[a], w[a]);
      b[3 + a] = std::max(b[3 + a], w[a]);
    }
  }
  bounds = {{b[0], b[1], b[2]}, {b[3], b[4], b[5]}};
}

// verifyTemporalData (common/temporal_data_verification.h:10-181): the
// reference's checks and messages; returns the number of data elements the
// temporal format implies.
uint64_t verifyTemporalData(uint64_t numVoxels, uint32_t format, int numTimesteps, Data *indices, Data *times)
{
  if (format == 0) {
    if (numTimesteps != 0)
      fail("Temporally constant volumes should not have temporallyStructuredNumTimesteps provided");
    if (indices || times)
      fail("Temporally constant volumes should not have temporallyUnstructuredIndices or "
           "temporallyUnstructuredTimes provided");
    return numVoxels;
  }
  if (format == 1) {
    if (indices || times)
      fail("Temporally structured volumes should not have temporallyUnstructuredIndices or "
           "temporallyUnstructuredTimes provided");
    return numVoxels * (uint64_t)numTimesteps;
  }
  if (numTimesteps != 0)
    fail("Temporally unstructured volumes should not have temporallyStructuredNumTimesteps provided");
  if (!times)
    fail("temporal format is VKL_TEMPORAL_FORMAT_UNSTRUCTURED but temporallyUnstructuredTimes is not "
         "specified.");
  if (indices->numItems < numVoxels + 1)
    fail("temporallyUnstructuredIndices is too small.");
  const bool need64 = numVoxels >= (uint64_t)std::numeric_limits<uint32_t>::max();
  if (need64 && indices->type != VKL_ULONG)
    fail("temporallyUnstructuredIndices must be VKL_ULONG due to attribute data size");
  if (indices->type != VKL_UINT && indices->type != VKL_ULONG)
    fail("temporallyUnstructuredIndices must have type VKL_UINT or VKL_ULONG");
  if (times->type != VKL_FLOAT)
    fail("temporallyUnstructuredIndices must have type VKL_FLOAT");
  const uint8_t *ib = indices->hostBytes();
  const float *t    = (const float *)times->hostBytes();
  auto at           = [&](uint64_t i) -> uint64_t {
    if (indices->type == VKL_ULONG) {
      uint64_t v;
      std::memcpy(&v, ib + 8 * i, 8);
      return v;
    }
    uint32_t v;
    std::memcpy(&v, ib + 4 * i, 4);
    return v;
  };
  uint64_t b = 0, e = 0;
  for (uint64_t i = 0; i < numVoxels; ++i) {
    b = at(i);
    e = at(i + 1);
    if (!(b < e))
      fail("temporallyUnstructuredIndices must increase strictly monotonically.");
    if (!(e <= times->numItems))
      fail("Values in temporallyUnstructuredIndices are out of bounds in temporallyUnstructredTimes.");
    for (uint64_t k = b + 1; k < e; ++k)
      if (!(t[k - 1] < t[k]))
        fail("temporallyUnstructuredTimes must increase strictly monotonically for every voxel.");
    if (t[b] < 0.f || t[b] > 1.f || t[e - 1] < 0.f || t[e - 1] > 1.f)
      fail("Values in temporallyUnstructuredTimes must be bounded by 0.0 and 1.0 for every voxel.");
  }
  return e;
}

void Volume::commitDense()
{
  const int zero3[3] = {0, 0, 0};
  int dims[3];
  if (!has("dimensions"))
    fail("structuredRegular: missing required 'dimensions' parameter");
  getVec3i("dimensions", dims, zero3);
  const float zf3[3] = {0, 0, 0}, s1[3] = {1, 1, 1};
  float go[3], gs[3];
  getVec3f("gridOrigin", go, zf3);
  getVec3f("gridSpacing", gs, s1);
  int io[3];
  getVec3i("indexOrigin", io, zero3);
  std::vector<Data *> attrs = attributeArrays(*this, "data");
  if (attrs.empty())
    fail("structuredRegular: missing required 'data' parameter");
  if (attrs.size() > kMaxAttributes)
    fail("too many attributes for the cuda device (max 16)");
  if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0)
    fail("Vdb volumes must have at least one leaf node.");
  const uint64_t nvox = (uint64_t)dims[0] * dims[1] * dims[2];
  for (size_t i = 0; i < attrs.size(); ++i)
    if (!isVoxelType(attrs[i]->type))
      fail("structuredRegular: unsupported data element type (attribute " + std::to_string(i) +
               ") for 'data' parameter");
  // Motion-blur data (DenseVdbVolume.cpp:149-186): the temporal format
  // follows from which parameters are present, and the data arrays must
  // hold the number of elements it implies.
  const int numTimesteps = getInt("temporallyStructuredNumTimesteps", 0);
  Data *tIdx             = getData("temporallyUnstructuredIndices");
  Data *tTimes           = getData("temporallyUnstructuredTimes");
  const uint32_t temporal = numTimesteps > 0 ? 1u : (tIdx ? 2u : 0u);
  const uint64_t expectedItems = verifyTemporalData(nvox, temporal, numTimesteps, tIdx, tTimes);
  for (size_t i = 0; i < attrs.size(); ++i)
    if (attrs[i]->numItems != expectedItems)
      fail("attribute " + std::to_string(i) + " has " + std::to_string(attrs[i]->numItems) +
               " elements, but expected " + std::to_string(expectedItems));

  grid.dense            = 1;
  grid.constantCellData = getBool("cellCentered", false) ? 1 : 0;
  grid.numAttributes    = (uint32_t)attrs.size();
  for (int a = 0; a < 3; ++a) {
    grid.denseDims[a]  = dims[a];
    grid.rootOrigin[a] = io[a];
    grid.activeSize[a] = (uint32_t)dims[a];
  }
  float c[12];
  if (!readIndexToObject(*this, c)) {
    const float cc[12] = {gs[0], 0, 0, 0, gs[1], 0, 0, 0, gs[2], go[0], go[1], go[2]};
    std::memcpy(c, cc, sizeof(c));
  }
  makeTransforms(c, grid.indexToObject, grid.objectToIndex);
  // background: one value, or one per attribute (ManagedObject.h:59-66)
  {
    std::vector<float> bg(grid.numAttributes, undefinedBackground());
    Data *bd = getData("background");
    if (bd) {
      const float *v = bd->hostAs<float>();
      if (bd->numItems == 1)
        std::fill(bg.begin(), bg.end(), v[0]);
      else if (bd->numItems == grid.numAttributes)
        std::copy(v, v + bd->numItems, bg.begin());
      else
        fail("background has the wrong number of elements");
    } else if (has("background")) {
      std::fill(bg.begin(), bg.end(), getFloat("background", bg[0]));
    }
    std::copy(bg.begin(), bg.end(), grid.background);
  }

  // Index box: [origin, origin+dims-1] vertex-centered, +dims cell-centered.
  const int e = grid.constantCellData ? 0 : 1;
  const float lo[3] = {(float)io[0], (float)io[1], (float)io[2]};
  const float hi[3] = {(float)(io[0] + dims[0] - e), (float)(io[1] + dims[1] - e),
                       (float)(io[2] + dims[2] - e)};
  finishCommit(lo, hi);

  // Tree: leaves of 8^3, level-2 nodes of 128^3, level-1 nodes of 4096^3.
  uint32_t nl[3], n2[3], n1[3];
  for (int a = 0; a < 3; ++a) {
    nl[a] = (uint32_t)((dims[a] + 7) / 8);
    n2[a] = (nl[a] + 15) / 16;
    n1[a] = (n2[a] + 31) / 32;
  }
  if (n1[0] > 64 || n1[1] > 64 || n1[2] > 64)
    fail("input leaves do not fit into a single root level node");
  const uint64_t N2 = (uint64_t)n2[0] * n2[1] * n2[2], N1 = (uint64_t)n1[0] * n1[1] * n1[2];
  grid.numLeaves    = (uint64_t)nl[0] * nl[1] * nl[2];
  const uint64_t NA = grid.numAttributes;
  DeviceBuffer *v0 = newBuffer(262144 * 8), *v1 = newBuffer(N1 * 32768 * 8),
               *v2 = newBuffer(N2 * 4096 * 8);
  DeviceBuffer *o1 = newBuffer(N1 * 12), *o2 = newBuffer(N2 * 12), *o0 = newBuffer(12);
  DeviceBuffer *r0 = newBuffer(262144 * 8 * NA), *r1 = newBuffer(N1 * 32768 * 8 * NA),
               *r2 = newBuffer(N2 * 4096 * 8 * NA);
  cudaStream_t st = device->stream;
  cudaCheck(cudaMemsetAsync(o0->ptr, 0, 12, st), "memset");
  grid.levels[0] = {1, o0->as<uint32_t>(), v0->as<uint64_t>(), r0->as<float>()};
  grid.levels[1] = {N1, o1->as<uint32_t>(), v1->as<uint64_t>(), r1->as<float>()};
  grid.levels[2] = {N2, o2->as<uint32_t>(), v2->as<uint64_t>(), r2->as<float>()};
  levelNodes[0] = 1;
  levelNodes[1] = N1;
  levelNodes[2] = N2;
  levelNodes[3] = grid.numLeaves;
  launchBuildDenseTree(grid, v0->as<uint64_t>(), v1->as<uint64_t>(), v2->as<uint64_t>(),
                       o1->as<uint32_t>(), o2->as<uint32_t>(), nl, n1, n2, st);

  // Each attribute is re-laid out once into the bricked order the kernels
  // read (grid.h brickIndex) by the same pass that computes its leaf ranges.
  // The padding of partial supertiles is zeroed and never read (every tap is
  // checked against the domain first).
  // leaf ranges and the volume range: scratch of the commit, kept with the
  // volume so that a re-commit reuses them
  // volRange also holds one denormal flag per attribute after the ranges.
  DeviceBuffer &leafRanges = *newBuffer(grid.numLeaves * 8), &volRange = *newBuffer(12 * NA);
  uint32_t *denormalFlags  = (uint32_t *)(volRange.as<float>() + 2 * NA);
  cudaCheck(cudaMemsetAsync(denormalFlags, 0, 4 * NA, st), "memset");
  if (temporal) {
    // the data stay as given (x fastest, time samples consecutive): no
    // bricked copy and no texture atlas
    grid.temporal     = temporal;
    grid.numTimesteps = (uint32_t)std::max(numTimesteps, 0);
    if (temporal == 2) {
      keep.emplace_back(tIdx);
      keep.emplace_back(tTimes);
      grid.tIndices = tIdx->dev;
      grid.tIndex64 = tIdx->type == VKL_ULONG ? 1u : 0u;
      grid.tTimes   = (const float *)tTimes->dev;
    }
    for (uint32_t a = 0; a < NA; ++a) {
      keep.emplace_back(attrs[a]);
      grid.data[a] = attrs[a]->dev;
      grid.type[a] = attrs[a]->type;
      if (atlases[a])
        device->giveAtlas(std::move(atlases[a]));
      launchTemporalLeafRanges(grid, a, nl, leafRanges.as<float>(), st);
      launchPropagateRanges(grid, a, grid.numLeaves, nullptr, leafRanges.as<float>(),
                            volRange.as<float>() + 2 * a, nl, st);
    }
    std::vector<float> vr(3 * NA);
    cudaCheck(cudaMemcpyAsync(vr.data(), volRange.ptr, 12 * NA, cudaMemcpyDeviceToHost, st),
              "value range readback");
    cudaCheck(cudaStreamSynchronize(st), "dense commit");
    rangeLo.assign(NA, 0);
    rangeHi.assign(NA, 0);
    for (uint32_t a = 0; a < NA; ++a) {
      rangeLo[a] = vr[2 * a];
      rangeHi[a] = vr[2 * a + 1];
    }
    return;
  }
  const uint32_t udims[3] = {(uint32_t)dims[0], (uint32_t)dims[1], (uint32_t)dims[2]};
  const uint64_t nb       = brickedElements(udims, grid.superX, grid.superY);
  // Texture atlases of float attributes (trilinear sampling through tld4):
  // planes side by side, written by the commit pass itself.
  const uint32_t planesPerRow =
      device->textureSampling ? atlasPlanesPerRow(device->cudaDevice, udims[0], udims[1], udims[2]) : 0;
  grid.atlasPlanesPerRow = planesPerRow ? planesPerRow : 1;
  for (uint32_t a = 0; a < grid.numAttributes; ++a) {
    const size_t es  = sizeOfType(attrs[a]->type);
    DeviceBuffer *bb = newBuffer(nb * es);
    if (nb != nvox)
      cudaCheck(cudaMemsetAsync(bb->ptr, 0, nb * es, st), "memset");
    grid.data[a] = bb->ptr;
    grid.type[a] = attrs[a]->type;
    uint64_t surf = 0;
    if (planesPerRow && attrs[a]->type == VKL_FLOAT) {
      const uint32_t w = planesPerRow * udims[0], h = (udims[2] + planesPerRow - 1) / planesPerRow * udims[1];
      if (atlases[a] && (atlases[a]->width != w || atlases[a]->height != h))
        device->giveAtlas(std::move(atlases[a]));
      if (!atlases[a])
        atlases[a] = device->takeAtlas(w, h);
      if (!atlases[a])
        atlases[a].reset(new TextureAtlas());
      bool ok = atlases[a]->ensure(w, h);
      if (!ok) {  // memory held by pooled atlases first
        device->dropAtlases();
        ok = atlases[a]->ensure(w, h);
      }
      if (ok)
        surf = atlases[a]->surf;
    } else if (atlases[a]) {
      device->giveAtlas(std::move(atlases[a]));
    }
    launchDenseBrickRanges(attrs[a]->dev, attrs[a]->type, bb->ptr, udims, grid.superX, grid.superY,
                           grid.background[a], leafRanges.as<float>(), surf, grid.atlasPlanesPerRow,
                           denormalFlags + a, st);
    launchPropagateRanges(grid, a, grid.numLeaves, nullptr, leafRanges.as<float>(),
                          volRange.as<float>() + 2 * a, nl, st);
  }
  std::vector<float> vr(3 * NA);
  cudaCheck(cudaMemcpyAsync(vr.data(), volRange.ptr, 12 * NA, cudaMemcpyDeviceToHost, st),
            "value range readback");
  cudaCheck(cudaStreamSynchronize(st), "dense commit");
  // an attribute with denormal voxels is sampled without its atlas (the
  // texture path would flush them to zero)
  for (uint32_t a = 0; a < NA; ++a) {
    uint32_t denormal = 0;
    std::memcpy(&denormal, &vr[2 * NA + a], 4);
    if (atlases[a] && atlases[a]->array && !denormal)
      grid.atlasTex[a] = atlases[a]->tex;
    else if (atlases[a])
      device->giveAtlas(std::move(atlases[a]));
  }
  rangeLo.assign(NA, 0);
  rangeHi.assign(NA, 0);
  for (uint32_t a = 0; a < NA; ++a) {
    rangeLo[a] = vr[2 * a];
    rangeHi[a] = vr[2 * a + 1];
  }
}

void Volume::commitVdb()
{
  Data *dLevel  = getData("node.level");
  Data *dOrigin = getData("node.origin");
  Data *dFormat = getData("node.format");
  const bool hasNodeData = getData("node.data") != nullptr;
  const bool hasPacked   = getData("nodesPackedDense") != nullptr;
  if (hasNodeData && hasPacked)
    fail("provide either node.data or nodesPackedDense / nodesPackedTile, not both");
  if (!hasNodeData && !hasPacked)
    fail("node.data or nodesPackedDense / nodesPackedTile must be provided");
  if (!dLevel || !dOrigin || !dFormat)
    fail("node.level, node.origin and node.format must be provided");
  const uint64_t numLeaves = dLevel->numItems;
  if (numLeaves == 0)
    fail("Vdb volumes must have at least one leaf node.");
  if (dOrigin->numItems != numLeaves || dFormat->numItems != numLeaves)
    fail("node.level, node.origin, node.format, node.temporalFormat, and node.data must all have "
         "the same size");
  if (Data *tf = getData("node.temporalFormat")) {
    if (tf->numItems != numLeaves)
      fail("node.level, node.origin, node.format, node.temporalFormat, and node.data must all have "
           "the same size");
    const uint32_t *t = tf->hostAs<uint32_t>();
    for (uint64_t i = 0; i < tf->numItems; ++i)
      if (t[i] != 0)
        fail("temporally varying (motion blur) volumes are not supported by the cuda device",
             VKL_INVALID_OPERATION);
  }
  // present with constant nodes: size-checked as the reference does
  // (VdbVolume.cpp:720-746), otherwise unused
  for (const char *name : {"node.temporallyStructuredNumTimesteps", "node.temporallyUnstructuredIndices",
                           "node.temporallyUnstructuredTimes"}) {
    Data *d = getData(name);
    if (d && d->numItems != numLeaves)
      fail(std::string("If ") + name + " is set, it must have the same size as node.data");
  }
  const uint32_t *levels = dLevel->hostAs<uint32_t>();
  const int32_t *origins = dOrigin->hostAs<int32_t>();
  const uint32_t *formats = dFormat->hostAs<uint32_t>();

  grid.dense            = 0;
  grid.constantCellData = 1;
  grid.numLeaves        = numLeaves;
  float c[12]           = {1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0};
  readIndexToObject(*this, c);
  makeTransforms(c, grid.indexToObject, grid.objectToIndex);

  // Leaf validation and packed indices (VdbVolume.cpp:850-994).
  std::vector<uint64_t> packedIndex(numLeaves);
  uint64_t nDense = 0, nTile = 0;
  for (uint64_t i = 0; i < numLeaves; ++i) {
    if (levels[i] >= kNumLevels)
      fail("invalid node level " + std::to_string(levels[i]) + " for this vdb configuration");
    if (levels[i] == 0)
      fail("there must not be any leaf nodes on level 0");
    if (formats[i] == kFormatDenseZYX) {
      if (levels[i] + 1 < kNumLevels)
        fail("leaf nodes are only supported on the lowest level.");
      packedIndex[i] = nDense++;
    } else if (formats[i] == kFormatTile) {
      packedIndex[i] = nTile++;
    } else {
      fail("invalid format specified");
    }
  }

  // Leaf storage: packed arrays used in place, node.data packed here into the
  // same layout indexed by the original leaf index.
  uint32_t leafType = 0;
  if (hasPacked) {
    std::vector<Data *> pd = attributeArrays(*this, "nodesPackedDense");
    std::vector<Data *> pt = attributeArrays(*this, "nodesPackedTile");
    grid.numAttributes     = (uint32_t)pd.size();
    if (grid.numAttributes == 0 || grid.numAttributes > kMaxAttributes)
      fail("nodesPackedDense must hold 1..16 attributes");
    if (!pt.empty() && pt.size() != pd.size())
      fail("nodesPackedTile must have one array per attribute");
    for (uint32_t a = 0; a < grid.numAttributes; ++a) {
      const VKLDataType t = pd[a]->type;
      if (t != VKL_HALF && t != VKL_FLOAT)
        fail("nodesPackedDense must be VKL_HALF or VKL_FLOAT");
      if (a == 0)
        leafType = t;
      else if (t != (VKLDataType)leafType)
        fail("nodesPackedDense has inconsistent attribute type");
      if (pd[a]->numItems != nDense * 512)
        fail("nodesPackedDense has incorrect number of elements");
      keep.emplace_back(pd[a]);
      grid.data[a] = pd[a]->dev;
      if (!pt.empty()) {
        if (pt[a]->type != (VKLDataType)leafType)
          fail("nodesPackedTile has inconsistent attribute type");
        if (pt[a]->numItems != nTile)
          fail("nodesPackedTile has incorrect number of elements");
        keep.emplace_back(pt[a]);
        grid.tile[a] = pt[a]->dev;
      } else if (nTile) {
        fail("nodesPackedTile must be provided for tile nodes");
      }
      grid.type[a] = leafType;
    }
  } else {
    Data *nd = getData("node.data");
    if (nd->numItems != numLeaves)
      fail("node.data has incorrect size");
    // per leaf: a Data (one attribute) or a Data of Data (attributes)
    std::vector<std::vector<Data *>> leafAttr(numLeaves);
    for (uint64_t i = 0; i < numLeaves; ++i) {
      Data *ld = dynamic_cast<Data *>(nd->objects[i]);
      if (!ld)
        fail("node.data holds a non-data object");
      if (ld->type == VKL_DATA) {
        for (ManagedObject *m : ld->objects)
          leafAttr[i].push_back(dynamic_cast<Data *>(m));
      } else {
        leafAttr[i].push_back(ld);
      }
    }
    grid.numAttributes = (uint32_t)leafAttr[0].size();
    if (grid.numAttributes == 0 || grid.numAttributes > kMaxAttributes)
      fail("node.data must hold 1..16 attributes");
    for (uint32_t a = 0; a < grid.numAttributes; ++a) {
      const VKLDataType t = leafAttr[0][a]->type;
      if (t != VKL_HALF && t != VKL_FLOAT)
        fail("node.data arrays must be VKL_HALF or VKL_FLOAT");
      if (a == 0)
        leafType = t;
      else if (t != (VKLDataType)leafType)
        fail("All nodes must have the same VKLDataType in vdb volumes.");
    }
    const size_t ts = sizeOfType((VKLDataType)leafType);
    for (uint32_t a = 0; a < grid.numAttributes; ++a) {
      std::vector<uint8_t> dense(numLeaves * 512 * ts, 0), tile(numLeaves * ts, 0);
      for (uint64_t i = 0; i < numLeaves; ++i) {
        if (leafAttr[i].size() != grid.numAttributes || !leafAttr[i][a])
          fail("inconsistent leaf attribute count");
        Data *d = leafAttr[i][a];
        if (d->type != (VKLDataType)leafType)
          fail("inconsistent leaf attribute data type");
        const uint64_t expect = formats[i] == kFormatTile ? 1 : 512;
        if (d->numItems < expect)
          fail("Node data too small: found " + std::to_string(d->numItems) +
                   " elements, but expected " + std::to_string(expect));
        if (d->numItems > expect)
          fail("Node data too big: found " + std::to_string(d->numItems) +
                   " elements, but expected " + std::to_string(expect));
        if (formats[i] == kFormatTile)
          std::memcpy(&tile[i * ts], d->hostBytes(), ts);
        else
          std::memcpy(&dense[i * 512 * ts], d->hostBytes(), 512 * ts);
      }
      DeviceBuffer *bd = newBuffer(dense.size()), *bt = newBuffer(tile.size());
      cudaCheck(cudaMemcpy(bd->ptr, dense.data(), dense.size(), cudaMemcpyHostToDevice), "upload");
      cudaCheck(cudaMemcpy(bt->ptr, tile.data(), tile.size(), cudaMemcpyHostToDevice), "upload");
      grid.data[a] = bd->ptr;
      grid.tile[a] = bt->ptr;
      grid.type[a] = leafType;
    }
  }
  // Compressed leaves (extension parameter "compression": "fp16" | "bf16" |
  // "fp8"): float packed leaves are re-encoded on the GPU with one
  // (scale, offset) pair per leaf; tiles stay float.  The stencil-block
  // forms ("fp16_blocks" | "bf16_blocks" | "fp8_blocks") are encoded after
  // the tree and leaf map exist (their blocks reach into neighbouring leaves).
  uint32_t blockedFmt = kCompressNone;
  if (const Param *cp = find("compression")) {
    const std::string &c = cp->str;
    uint32_t fmt = kCompressNone;
    if (c == "fp16")
      fmt = kCompressFP16;
    else if (c == "bf16")
      fmt = kCompressBF16;
    else if (c == "fp8" || c == "fp8_e4m3")
      fmt = kCompressFP8;
    else if (c == "fp16_blocks")
      blockedFmt = kCompressFP16Blocks;
    else if (c == "bf16_blocks")
      blockedFmt = kCompressBF16Blocks;
    else if (c == "fp8_blocks" || c == "fp8_e4m3_blocks")
      blockedFmt = kCompressFP8Blocks;
    else if (!(c.empty() || c == "none"))
      fail("compression must be one of none, fp16, bf16, fp8, fp16_blocks, bf16_blocks, fp8_blocks");
    if (blockedFmt != kCompressNone && leafType != VKL_FLOAT)
      fail("compression requires VKL_FLOAT leaves");
    if (fmt != kCompressNone) {
      if (leafType != VKL_FLOAT)
        fail("compression requires VKL_FLOAT leaves");
      const uint64_t slots   = hasPacked ? nDense : numLeaves;
      const size_t codeBytes = fmt == kCompressFP8 ? 1 : 2;
      for (uint32_t a = 0; a < grid.numAttributes; ++a) {
        DeviceBuffer *bc = newBuffer(std::max<uint64_t>(slots, 1) * 512 * codeBytes);
        DeviceBuffer *bs = newBuffer(std::max<uint64_t>(slots, 1) * 8);
        launchCompressLeaves(fmt, (const float *)grid.data[a], slots, bc->ptr, bs->as<float>(),
                             device->stream);
        grid.data[a]            = bc->ptr;
        grid.leafScaleOffset[a] = bs->as<float>();
      }
      cudaCheck(cudaStreamSynchronize(device->stream), "leaf compression");
    }
    grid.compress = fmt;
  }
  {
    std::vector<float> bg(grid.numAttributes, undefinedBackground());
    Data *bd = getData("background");
    if (bd) {
      const float *v = bd->hostAs<float>();
      if (bd->numItems == 1)
        std::fill(bg.begin(), bg.end(), v[0]);
      else if (bd->numItems == grid.numAttributes)
        std::copy(v, v + bd->numItems, bg.begin());
      else
        fail("background has the wrong number of elements");
    } else if (has("background")) {
      std::fill(bg.begin(), bg.end(), getFloat("background", bg[0]));
    }
    std::copy(bg.begin(), bg.end(), grid.background);
  }

  // Bounding box and root origin (VdbVolume.cpp:71-81, :567-581, :766-806).
  int64_t lo[3] = {INT64_MAX, INT64_MAX, INT64_MAX}, hi[3] = {INT64_MIN, INT64_MIN, INT64_MIN};
  for (uint64_t i = 0; i < numLeaves; ++i) {
    const int64_t r = levelRes(levels[i]);
    for (int a = 0; a < 3; ++a) {
      const int64_t o = origins[3 * i + a];
      lo[a]           = std::min(lo[a], std::min(o, o + r));
      hi[a]           = std::max(hi[a], std::max(o, o + r));
    }
  }
  for (int a = 0; a < 3; ++a)
    if ((uint32_t)(hi[a] - lo[a]) > levelRes(0))
      fail("input leaves do not fit into a single root level node");
  const int32_t r1 = (int32_t)levelRes(1);
  for (int a = 0; a < 3; ++a) {
    grid.rootOrigin[a] = r1 * (int32_t)std::floor((float)lo[a] / (float)r1);
    grid.activeSize[a] = (uint32_t)(hi[a] - grid.rootOrigin[a]);
  }
  float flo[3] = {(float)lo[0], (float)lo[1], (float)lo[2]};
  float fhi[3] = {(float)hi[0], (float)hi[1], (float)hi[2]};
  if (const Param *p = find("indexClippingBounds")) {
    if (p->type == VKL_BOX3I) {
      int32_t b[6];
      std::memcpy(b, p->bytes.data(), 24);
      if (!(b[3] < b[0] || b[4] < b[1] || b[5] < b[2]))
        for (int a = 0; a < 3; ++a) {
          flo[a] = (float)b[a];
          fhi[a] = (float)b[3 + a];
        }
    }
  }
  finishCommit(flo, fhi);

  // Tree insertion (VdbVolume.cpp:86-331): count distinct nodes per level
  // bottom-up, then insert leaves level-binned in input order, numbering new
  // nodes first-come.
  std::vector<uint32_t> off(3 * numLeaves);
  for (uint64_t i = 0; i < numLeaves; ++i)
    for (int a = 0; a < 3; ++a)
      off[3 * i + a] = (uint32_t)(origins[3 * i + a] - grid.rootOrigin[a]);
  std::vector<std::vector<uint64_t>> binned(kNumLevels);
  for (uint64_t i = 0; i < numLeaves; ++i)
    binned[levels[i]].push_back(i);
  uint64_t capacity[kNumLevels - 1] = {0, 0, 0};
  {
    std::unordered_set<uint64_t> prev;
    std::vector<uint64_t> prevList;
    for (int l = kNumLevels - 1; l >= 1; --l) {
      const uint32_t mask = ~(levelRes(l - 1) - 1);
      std::unordered_set<uint64_t> cur;
      std::vector<uint64_t> curList;
      auto add = [&](uint32_t x, uint32_t y, uint32_t z) {
        const uint64_t k = packKey(x & mask, y & mask, z & mask);
        if (cur.insert(k).second)
          curList.push_back(k);
      };
      for (uint64_t leaf : binned[l])
        add(off[3 * leaf], off[3 * leaf + 1], off[3 * leaf + 2]);
      for (uint64_t k : prevList)
        add((uint32_t)(k >> 42), (uint32_t)((k >> 21) & 0x1fffff), (uint32_t)(k & 0x1fffff));
      capacity[l - 1] = curList.size();
      prev.swap(cur);
      prevList.swap(curList);
    }
  }
  std::vector<uint64_t> vox[kNumLevels - 1];
  std::vector<uint32_t> org[kNumLevels - 1];
  uint64_t numNodes[kNumLevels - 1] = {1, 0, 0};
  for (uint32_t l = 0; l < kNumLevels - 1; ++l) {
    vox[l].assign(std::max<uint64_t>(capacity[l], l == 0 ? 1 : 0) * levelNumVoxels(l), 0);
    org[l].assign(3 * std::max<uint64_t>(capacity[l], l == 0 ? 1 : 0), 0);
  }
  std::vector<uint64_t> leafVoxel(numLeaves, ~0ull);
  for (uint32_t leafLevel = 0; leafLevel < kNumLevels; ++leafLevel)
    for (uint64_t idx : binned[leafLevel]) {
      const uint32_t ox = off[3 * idx], oy = off[3 * idx + 1], oz = off[3 * idx + 2];
      uint64_t node = 0;
      for (uint32_t l = 0; l < leafLevel; ++l) {
        const uint64_t v = node * levelNumVoxels(l) + offsetToLinear(l, ox, oy, oz);
        uint64_t &voxel  = vox[l][v];
        if (voxelIsLeaf(voxel)) {
          fail("Attempted to insert a leaf node into a leaf node (level " + std::to_string(l + 1) +
                   ")");
        } else if (voxelIsEmpty(voxel)) {
          const uint32_t nl = l + 1;
          if (nl < leafLevel) {
            node  = numNodes[nl]++;
            voxel = voxelMakeChild(node);
            const uint32_t m = ~(levelRes(nl) - 1);
            org[nl][3 * node]     = ox & m;
            org[nl][3 * node + 1] = oy & m;
            org[nl][3 * node + 2] = oz & m;
          } else {
            voxel          = voxelMakeLeaf(hasPacked ? packedIndex[idx] : idx, formats[idx], 0);
            leafVoxel[idx] = ((uint64_t)l << 40) | v;
          }
        } else {
          node = voxelChildIndex(voxel);
        }
      }
    }
  const uint64_t NA = grid.numAttributes;
  cudaStream_t st   = device->stream;
  for (uint32_t l = 0; l < kNumLevels - 1; ++l) {
    levelNodes[l]     = numNodes[l];
    DeviceBuffer *bv = newBuffer(vox[l].size() * 8);
    DeviceBuffer *bo = newBuffer(org[l].size() * 4);
    DeviceBuffer *br = newBuffer(vox[l].size() * 8 * NA);
    if (!vox[l].empty()) {
      cudaCheck(cudaMemcpy(bv->ptr, vox[l].data(), vox[l].size() * 8, cudaMemcpyHostToDevice),
                "upload");
      cudaCheck(cudaMemcpy(bo->ptr, org[l].data(), org[l].size() * 4, cudaMemcpyHostToDevice),
                "upload");
    }
    grid.levels[l] = {numNodes[l], bo->as<uint32_t>(), bv->as<uint64_t>(), br->as<float>()};
  }
  levelNodes[3] = numLeaves;

  // Flat leaf map (sampling replaces the walk by one load) when it fits its
  // budget; parameter "leafMap" (bool, default true) turns it off.
  {
    uint64_t slots = 1;
    for (int a = 0; a < 3; ++a) {
      grid.leafMapDims[a] = (grid.activeSize[a] + 7) / 8;
      slots *= grid.leafMapDims[a];
    }
    if (getBool("leafMap", true) && slots * 8 <= kLeafMapBudgetBytes) {
      DeviceBuffer *bm = newBuffer(std::max<uint64_t>(slots, 1) * 8);
      launchBuildLeafMap(grid, bm->as<uint64_t>(), device->stream);
      grid.leafMap = bm->as<uint64_t>();
    } else {
      grid.leafMapDims[0] = grid.leafMapDims[1] = grid.leafMapDims[2] = 0;
    }
  }

  if (blockedFmt != kCompressNone) {
    // per dense slot its leaf's root-relative offset (~0: a tile's unused
    // slot of node.data input)
    const uint64_t slots = hasPacked ? nDense : numLeaves;
    std::vector<uint32_t> slotOff(3 * std::max<uint64_t>(slots, 1), ~0u);
    for (uint64_t i = 0; i < numLeaves; ++i)
      if (formats[i] == kFormatDenseZYX) {
        const uint64_t sl = hasPacked ? packedIndex[i] : i;
        for (int a = 0; a < 3; ++a)
          slotOff[3 * sl + a] = off[3 * i + a];
      }
    DeviceBuffer dSlotOff;
    dSlotOff.alloc(slotOff.size() * 4);
    cudaCheck(cudaMemcpy(dSlotOff.ptr, slotOff.data(), slotOff.size() * 4, cudaMemcpyHostToDevice), "upload");
    const size_t codeBytes = blockedFmt == kCompressFP8Blocks ? 1 : 2;
    const DevGrid floatGrid = grid;
    for (uint32_t a = 0; a < grid.numAttributes; ++a) {
      DeviceBuffer *bc = newBuffer(std::max<uint64_t>(slots, 1) * kLeafCodes * codeBytes);
      DeviceBuffer *bs = newBuffer(std::max<uint64_t>(slots, 1) * 8);
      launchBuildLeafBlocks(blockedFmt, floatGrid, a, slots, dSlotOff.as<uint32_t>(), bc->ptr, bs->as<float>(),
                            device->stream);
      grid.data[a]            = bc->ptr;
      grid.leafScaleOffset[a] = bs->as<float>();
    }
    cudaCheck(cudaStreamSynchronize(device->stream), "leaf blocks");
    grid.compress = blockedFmt;
  }

  DeviceBuffer dOff, dLeafVoxel, leafRanges, volRange;
  dOff.alloc(off.size() * 4);
  dLeafVoxel.alloc(numLeaves * 8);
  leafRanges.alloc(numLeaves * 8);
  volRange.alloc(8 * NA);
  cudaCheck(cudaMemcpy(dOff.ptr, off.data(), off.size() * 4, cudaMemcpyHostToDevice), "upload");
  cudaCheck(cudaMemcpy(dLeafVoxel.ptr, leafVoxel.data(), numLeaves * 8, cudaMemcpyHostToDevice),
            "upload");
  const uint32_t nlDummy[3] = {0, 0, 0};
  for (uint32_t a = 0; a < NA; ++a) {
    launchSparseLeafRanges(grid, a, numLeaves, dOff.as<uint32_t>(), leafRanges.as<float>(), st);
    launchPropagateRanges(grid, a, numLeaves, dLeafVoxel.as<uint64_t>(), leafRanges.as<float>(),
                          volRange.as<float>() + 2 * a, nlDummy, st);
  }
  std::vector<float> vr(2 * NA);
  cudaCheck(cudaMemcpyAsync(vr.data(), volRange.ptr, 8 * NA, cudaMemcpyDeviceToHost, st),
            "value range readback");
  cudaCheck(cudaStreamSynchronize(st), "vdb commit");
  rangeLo.assign(NA, 0);
  rangeHi.assign(NA, 0);
  for (uint32_t a = 0; a < NA; ++a) {
    rangeLo[a] = vr[2 * a];
    rangeHi[a] = vr[2 * a + 1];
  }
}

// ---------------------------------------------------------------------------
// Sampler (VdbSampler.cpp:37-60): the sampler's parameters override the
// volume's; gradientFilter falls back to the sampler's filter if that is set.
// ---------------------------------------------------------------------------
void Sampler::commit()
{
  if (!volume || !volume->committed)
    fail("sampler volume is not committed", VKL_INVALID_OPERATION);
  s.filter         = getInt("filter", volume->filter);
  s.gradientFilter = getInt("gradientFilter", has("filter") ? s.filter : volume->gradientFilter);
  s.maxSamplingDepth =
      (uint32_t)getInt("maxSamplingDepth", (int)volume->maxSamplingDepth);
  for (int f : {s.filter, s.gradientFilter})
    if (f != kFilterNearest && f != kFilterLinear && f != kFilterCubic)
      fail("invalid filter");
  uploadState();
}

DevGrid Sampler::launchGrid() const
{
  DevGrid g       = volume->grid;
  g.numLeafAccess = 0;
  for (Observer *o : leafObservers)
    if (g.numLeafAccess < kMaxLeafObservers)
      g.leafAccess[g.numLeafAccess++] = o->devCounters.as<uint32_t>();
  return g;
}

void Sampler::uploadState()
{
  // the handle's device pointer stays valid across commits: allocate once
  const DevSamplerState state{launchGrid(), s};
  if (!devState.ptr)
    devState.alloc(sizeof(state));
  cudaCheck(cudaMemcpy(devState.ptr, &state, sizeof(state), cudaMemcpyHostToDevice), "upload");
}

// ---------------------------------------------------------------------------
// Iterator contexts (IteratorContext.cpp:49-336).
// ---------------------------------------------------------------------------
static uint32_t hintToDepth(float hint)
{
  hint = std::max(std::min(1.f, hint), 0.f);
  const float th[4] = {0.f, 0.2f, 0.4f, 0.8f};
  int depth         = 0;
  for (int i = 0; i < 4; ++i) {
    if (hint >= th[i])
      depth = i;
    else
      break;
  }
  return (uint32_t)depth;
}

static void minMaxOf(const std::vector<float> &r, float mm[2])
{
  mm[0] = INFINITY;
  mm[1] = -INFINITY;
  for (size_t i = 0; i + 1 < r.size(); i += 2) {
    mm[0] = r[i] < mm[0] ? r[i] : mm[0];
    mm[1] = r[i + 1] > mm[1] ? r[i + 1] : mm[1];
  }
}

void IntervalContext::commit()
{
  if (!sampler)
    fail("interval iterator context has no sampler", VKL_INVALID_OPERATION);
  attr = (uint32_t)getInt("attributeIndex", 0);
  if (attr >= sampler->volume->grid.numAttributes)
    fail("invalid attributeIndex");
  ranges.clear();
  if (Data *d = getData("valueRanges")) {
    if (d->type != VKL_BOX1F)
      fail("valueRanges must be VKL_BOX1F data");
    const float *v = d->hostAs<float>();
    ranges.assign(v, v + 2 * d->numItems);
  }
  minMaxOf(ranges, minMax);
  macrocells = getBool("macrocells", false);
  if (macrocells) {
    checkMacrocellVolume(sampler->volume->grid);
    sampler->volume->macrocellRanges(attr, device->stream);
  }
  const float hint = getFloat("intervalResolutionHint", 0.5f);
  depth            = hintToDepth(hint);
  elementary       = std::max(std::min(1.f, hint), 0.f) == 1.f;
  devRanges.alloc(std::max<size_t>(8, ranges.size() * 4));
  if (!ranges.empty())
    cudaCheck(cudaMemcpy(devRanges.ptr, ranges.data(), ranges.size() * 4, cudaMemcpyHostToDevice),
              "upload");
  const DevIntervalContextState state{sampler->devState.as<DevSamplerState>(), devValueRanges(), attr,
                                      depth};
  if (!devState.ptr)
    devState.alloc(sizeof(state));
  cudaCheck(cudaMemcpy(devState.ptr, &state, sizeof(state), cudaMemcpyHostToDevice), "upload");
}

const float *Volume::macrocellRanges(uint32_t attr, cudaStream_t st)
{
  if (!macroRanges[attr]) {
    std::unique_ptr<DeviceBuffer> b(new DeviceBuffer());
    b->alloc(macrocellRangeCount(grid) * 8);
    launchMacrocellRanges(grid, attr, b->as<float>(), st);
    macroRanges[attr] = std::move(b);
  }
  return macroRanges[attr]->as<float>();
}

DevValueRanges IntervalContext::devValueRanges() const
{
  return {(uint32_t)(ranges.size() / 2), {minMax[0], minMax[1]}, devRanges.as<float>()};
}

void HitContext::commit()
{
  if (!sampler)
    fail("hit iterator context has no sampler", VKL_INVALID_OPERATION);
  attr = (uint32_t)getInt("attributeIndex", 0);
  if (attr >= sampler->volume->grid.numAttributes)
    fail("invalid attributeIndex");
  values.clear();
  if (Data *d = getData("values")) {
    if (d->type != VKL_FLOAT)
      fail("values must be VKL_FLOAT data");
    const float *v = d->hostAs<float>();
    values.assign(v, v + d->numItems);
  }
  ranges.clear();
  for (float v : values) {
    ranges.push_back(v);
    ranges.push_back(v);
  }
  minMaxOf(ranges, minMax);
  // sparse VDB iterates elementary cells (hint 1.0), dense uses hint 0.5
  depth = sampler->volume->isDense ? hintToDepth(0.5f) : hintToDepth(1.f);
  devRanges.alloc(std::max<size_t>(8, ranges.size() * 4));
  devValues.alloc(std::max<size_t>(4, values.size() * 4));
  if (!values.empty()) {
    cudaCheck(cudaMemcpy(devRanges.ptr, ranges.data(), ranges.size() * 4, cudaMemcpyHostToDevice),
              "upload");
    cudaCheck(cudaMemcpy(devValues.ptr, values.data(), values.size() * 4, cudaMemcpyHostToDevice),
              "upload");
  }
  const DevHitContextState state{sampler->devState.as<DevSamplerState>(), devValueRanges(),
                                 devValues.as<float>(), (uint32_t)values.size(), attr, depth};
  if (!devState.ptr)
    devState.alloc(sizeof(state));
  cudaCheck(cudaMemcpy(devState.ptr, &state, sizeof(state), cudaMemcpyHostToDevice), "upload");
}

DevValueRanges HitContext::devValueRanges() const
{
  return {(uint32_t)(ranges.size() / 2), {minMax[0], minMax[1]}, devRanges.as<float>()};
}

// ---------------------------------------------------------------------------
// Observers.  InnerNode (VdbInnerNodeObserver.cpp:20-185): the node boxes
// and value ranges of all leaf-pointer voxels and of non-empty voxels at
// maxDepth, read back from the device tree.
// ---------------------------------------------------------------------------
Observer::~Observer()
{
  if (kind == "LeafNodeAccess" && sampler) {
    auto &v = sampler->leafObservers;
    v.erase(std::remove(v.begin(), v.end(), this), v.end());
    try {
      sampler->uploadState();
    } catch (...) {
    }
  }
}

void Observer::commit()
{
  if (kind == "LeafNodeAccess") {
    // VdbLeafAccessObserver::map: the buffer as the sampling left it
    leafAccess.resize(numElements);
    cudaCheck(cudaStreamSynchronize(device->stream), "observer");
    if (numElements)
      cudaCheck(cudaMemcpy(leafAccess.data(), devCounters.ptr, numElements * 4, cudaMemcpyDeviceToHost),
                "observer readback");
    return;
  }
  buffer.clear();
  numElements = 0;
  if (kind == "InnerNode") {
    const Volume &v     = *volume;
    const uint32_t maxD = (uint32_t)std::min(getInt("maxDepth", 1), (int)kNumLevels - 1);
    const uint32_t NA   = v.grid.numAttributes;
    elementFloats       = 6 + 2 * NA;
    for (uint32_t l = 0; l <= maxD && l + 1 < kNumLevels; ++l) {
      const DevLevel &L = v.grid.levels[l];
      const uint64_t nv = L.numNodes * levelNumVoxels(l);
      std::vector<uint64_t> vox(nv);
      std::vector<float> rng(nv * 2 * NA);
      std::vector<uint32_t> org(3 * L.numNodes);
      cudaCheck(cudaMemcpy(vox.data(), L.voxels, nv * 8, cudaMemcpyDeviceToHost), "readback");
      cudaCheck(cudaMemcpy(rng.data(), L.valueRange, rng.size() * 4, cudaMemcpyDeviceToHost),
                "readback");
      cudaCheck(cudaMemcpy(org.data(), L.origin, org.size() * 4, cudaMemcpyDeviceToHost),
                "readback");
      const uint32_t lr = logRes(l), res = 1u << lr, cell = levelRes(l + 1);
      for (uint64_t n = 0; n < L.numNodes; ++n)
        for (uint32_t x = 0; x < res; ++x)
          for (uint32_t y = 0; y < res; ++y)
            for (uint32_t z = 0; z < res; ++z) {
              const uint64_t vi = (n << (3 * lr)) + ((uint64_t)x << (2 * lr)) + ((uint64_t)y << lr) + z;
              const uint64_t voxel = vox[vi];
              if (!(voxelIsLeaf(voxel) || (l == maxD && !voxelIsEmpty(voxel))))
                continue;
              const float lo[3] = {(float)(v.grid.rootOrigin[0] + (int32_t)(org[3 * n] + cell * x)),
                                   (float)(v.grid.rootOrigin[1] + (int32_t)(org[3 * n + 1] + cell * y)),
                                   (float)(v.grid.rootOrigin[2] + (int32_t)(org[3 * n + 2] + cell * z))};
              const float hi[3] = {lo[0] + (float)cell, lo[1] + (float)cell, lo[2] + (float)cell};
              float b[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
              const float *M = v.grid.indexToObject;
              for (int i = 0; i < 8; ++i) {
                const float p[3] = {(i & 1) ? hi[0] : lo[0], (i & 2) ? hi[1] : lo[1],
                                    (i & 4) ? hi[2] : lo[2]};
                const float w[3] = {M[0] * p[0] + M[1] * p[1] + M[2] * p[2] + M[9],
                                    M[3] * p[0] + M[4] * p[1] + M[5] * p[2] + M[10],
                                    M[6] * p[0] + M[7] * p[1] + M[8] * p[2] + M[11]};
                for (int a = 0; a < 3; ++a) {
                  b[a]     = std::min(b[a], w[a]);
                  b[3 + a] = std::max(b[3 + a], w[a]);
                }
              }
              buffer.insert(buffer.end(), b, b + 6);
              for (uint32_t a = 0; a < NA; ++a) {
                buffer.push_back(rng[2 * (vi * NA + a)]);
                buffer.push_back(rng[2 * (vi * NA + a) + 1]);
              }
              ++numElements;
            }
    }
  } else {
    fail("unsupported observer type '" + kind + "'");
  }
}

}  // namespace vklcuda
