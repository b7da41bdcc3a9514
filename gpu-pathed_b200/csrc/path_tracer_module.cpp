// Python module `path_tracer`: the reference GUI's binding surface
// (bindings/path_tracer_bindings.cu:10-87) over the C ABI of libpathed.
//
//   RenderSession(width, height)      render_session.h:44-130, render_session.cu:55-117
//   SceneModel (per-session editor)    scene_model.h, scene_model.cu
//   Vec3, RenderState, RendererType, MaterialType, MaterialIndex
//
// Headless: init() takes no GL buffers (the two PBO handles are accepted and ignored) and
// RenderState.pbo is 0; getRadianceBuffer() returns the progressive radiance as a numpy
// array instead of a PBO. Frame sizes follow the reference's SppOptimizer
// (spp_optimizer.cpp:8-29: one sample after a reset, then as many samples as fit an 80 ms
// budget at the last frame's rate). Only the CUDA path-tracer backend exists: selecting the
// OptiX or normals renderer raises.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pathed.h"

namespace py = pybind11;

namespace {

// materials/types.h:5-11
// Metal (5) is this build's metallic-F0 Beckmann material; the reference's enum stops at None.
enum class MaterialType { Lambertian = 0, Mirror = 1, Glass = 2, Microfacet = 3, None = 4, Metal = 5 };
// scene_model.h:15-19
enum class RendererType { CUDA = 0, Optix = 1, Normals = 2 };

struct Vec3 {
    float v[3];
    float x() const { return v[0]; }
    float y() const { return v[1]; }
    float z() const { return v[2]; }
};

struct RenderState {
    bool isRendering;
    unsigned pbo;
};

struct MaterialIndex {
    MaterialType materialType;
    size_t index;
};

void check(pt_session* s, int rc) {
    if (rc != PT_OK) throw std::runtime_error(std::string("libpathed: ") + pt_last_error(s));
}

// Samples per frame for an 80 ms frame budget (spp_optimizer.cpp:8-29).
class SppOptimizer {
public:
    void track(int spp, float ms) {
        if (ms > 0.f) next_ = std::max(1, (int)std::floor(kBudgetMs * (spp / ms)));
    }
    int estimate() {
        if (reset_) {
            reset_ = false;
            return 1;
        }
        return next_;
    }
    void reset() { reset_ = true; }

private:
    static constexpr float kBudgetMs = 80.f;
    int next_ = 1;
    bool reset_ = false;
};

class Session;

// Editor of the session's scene. Every setter applies the edit and restarts progressive
// accumulation, as the reference's subscription callback does (render_session.cu:82-116).
class SceneModel {
public:
    explicit SceneModel(Session* s) : s_(s) {}

    RendererType getRendererType() const { return renderer_; }
    void setRendererType(RendererType t);
    void setColor(float r, float g, float b);
    Vec3 getColor() const;
    void setEmit(float r, float g, float b);
    Vec3 getEmit() const;
    float getIOR() const;
    void setIOR(float ior);
    float getAlpha() const;
    void setAlpha(float alpha);
    int getMaterialID() const { return material_id_; }
    void setMaterialID(int id) { material_id_ = id; }
    MaterialType getMaterialType() const;
    void setMaterialType(MaterialType t);
    void setLightPosition(float p);
    float getLightPosition() const { return light_position_; }
    Vec3 getCameraOrigin() const;
    void setCameraOrigin(float x, float y, float z);
    Vec3 getCameraTarget() const;
    void setCameraTarget(float x, float y, float z);
    Vec3 getCameraUp() const;
    void setCameraUp(float x, float y, float z);
    int getMaxDepth() const;
    void setMaxDepth(int d);
    bool getNextEventEstimation() const;
    void setNextEventEstimation(bool on);
    void zoomCamera(float ticks);
    int getSpp() const { return spp_; }
    void updateSpp(int spp) { spp_ = spp; }

private:
    struct Mat {
        int type;
        float albedo[3], emit[3], ior, alpha;
    };
    Mat material(int id) const;
    void apply(const Mat& m);
    void camera(float out[11]) const;
    void set_camera(const float c[11]);

    Session* s_;
    int material_id_ = -1;
    float light_position_ = -0.6f;  // scene.h:17 defaultLightPosition
    int spp_ = 0;
    RendererType renderer_ = RendererType::CUDA;
};

class Session {
public:
    Session(int width, int height, int config, uint64_t seed) : w_(width), h_(height), model_(this) {
        pt_session* s = nullptr;
        if (pt_create(width, height, &s) != PT_OK || !s) throw std::runtime_error("pt_create failed");
        s_ = s;
        check(s_, pt_load_config(s_, config, seed));
        loaded();
    }
    ~Session() {
        if (s_) pt_destroy(s_);
    }
    Session(const Session&) = delete;
    Session& operator=(const Session&) = delete;

    // RenderSession::init (render_session.cu:119-136): device resources are created here.
    RenderState init(py::args) {
        check(s_, pt_reset(s_));
        optimizer_.reset();
        initialised_ = true;
        return RenderState{false, 0u};
    }

    // RenderSession::renderAsync (render_session.h:59-69)
    RenderState renderAsync() {
        require_init();
        if (in_flight_) throw std::runtime_error("a frame is already in flight");
        const int spp = optimizer_.estimate();
        check(s_, pt_render_async(s_, spp));
        // the optimizer tracks the samples the frame rendered (RenderRecord::spp): one for
        // the normals G-buffer (g_buffer.cu:116)
        frame_spp_ = model_.getRendererType() == RendererType::Normals ? 1 : spp;
        in_flight_ = true;
        return RenderState{true, 0u};
    }

    // RenderSession::pollRender (render_session.h:71-118)
    RenderState pollRender() {
        require_init();
        if (!in_flight_) return RenderState{false, 0u};
        int done = 0;
        float ms = 0.f;
        check(s_, pt_poll(s_, &done, &ms));
        if (done) {
            in_flight_ = false;
            optimizer_.track(frame_spp_, ms);
            int spp = 0;
            check(s_, pt_get_spp(s_, &spp));
            model_.updateSpp(spp);
            snapshot(spp);
        }
        return RenderState{!done, 0u};
    }

    // pollRender's snapshot (render_session.h:87-101): the radiance buffer as EXR whenever
    // the accumulated spp crosses a power of two from 2 to 2^20. The reference always writes
    // out.exr in its working directory; here it is off until a path is set ("" turns it off).
    void setSnapshotPath(const std::string& path) { snapshot_ = path; }
    std::string getSnapshotPath() const { return snapshot_; }

    // RenderSession::hitTest (render_session.h:54-56, hit_test.cu:25-82)
    void hitTest(int x, int y) {
        require_init();
        finish();
        int mat = -1;
        check(s_, pt_hit_test(s_, x, y, &mat));
        model_.setMaterialID(mat);
    }

    // Renderer::getRadianceBuffer (renderer.cpp:20-42): H x W x 3, row 0 = image bottom
    py::array_t<float> getRadianceBuffer() {
        finish();
        py::array_t<float> out({h_, w_, 3});
        check(s_, pt_readback(s_, out.mutable_data(), (size_t)w_ * h_ * 3));
        return out;
    }

    // H x W x 4 display bytes (sRGB, the PBO contents of updateFramebuffer, framebuffer.cu:7-41)
    py::array_t<uint8_t> readbackRGBA8() {
        finish();
        py::array_t<uint8_t> out({h_, w_, 4});
        check(s_, pt_readback_rgba8(s_, out.mutable_data(), (size_t)w_ * h_ * 4));
        return out;
    }

    // The reference hard-codes scene 0 (render_session.cu:69); these select a generated
    // configuration or caller arrays instead. Both reset the selection and the accumulation.
    void loadScene(int config, uint64_t seed) {
        finish();
        check(s_, pt_load_config(s_, config, seed));
        loaded();
    }
    // SceneParameters::getSceneData(index) / getCamera(index) (scene.cu:14-218), which the
    // reference's RenderSession constructor loads for index 0 from ../scenes
    void loadReferenceScene(int index, const std::string& scenes_dir) {
        finish();
        check(s_, pt_load_reference_scene(s_, index, scenes_dir.c_str()));
        loaded();
    }
    void loadSceneArrays(py::array_t<float, py::array::c_style | py::array::forcecast> tri_vertices,
                         py::object tri_normals,
                         py::array_t<int, py::array::c_style | py::array::forcecast> tri_materials,
                         py::array_t<float, py::array::c_style | py::array::forcecast> spheres,
                         py::array_t<int, py::array::c_style | py::array::forcecast> sphere_materials,
                         py::array_t<int, py::array::c_style | py::array::forcecast> material_types,
                         py::array_t<float, py::array::c_style | py::array::forcecast> material_albedo,
                         py::array_t<float, py::array::c_style | py::array::forcecast> material_emit,
                         py::array_t<float, py::array::c_style | py::array::forcecast> material_ior,
                         py::array_t<float, py::array::c_style | py::array::forcecast> material_alpha,
                         py::object env_rgba) {
        finish();
        const py::ssize_t nt = tri_vertices.size() / 9, ns = spheres.size() / 4, nm = material_types.size();
        if (tri_vertices.size() != nt * 9 || tri_materials.size() != nt || spheres.size() != ns * 4 ||
            sphere_materials.size() != ns || material_albedo.size() != nm * 3 || material_emit.size() != nm * 3 ||
            material_ior.size() != nm || material_alpha.size() != nm)
            throw std::invalid_argument("inconsistent scene array sizes");
        pt_scene_desc d{};
        d.num_triangles = (int)nt;
        d.tri_vertices = tri_vertices.data();
        py::array_t<float, py::array::c_style | py::array::forcecast> normals;
        if (!tri_normals.is_none()) {
            normals = tri_normals.cast<py::array_t<float, py::array::c_style | py::array::forcecast>>();
            if (normals.size() != nt * 9) throw std::invalid_argument("tri_normals must hold 9 floats per triangle");
            d.tri_normals = normals.data();
        }
        d.tri_materials = tri_materials.data();
        d.num_spheres = (int)ns;
        d.spheres = spheres.data();
        d.sphere_materials = sphere_materials.data();
        d.num_materials = (int)nm;
        d.material_types = material_types.data();
        d.material_albedo = material_albedo.data();
        d.material_emit = material_emit.data();
        d.material_ior = material_ior.data();
        d.material_alpha = material_alpha.data();
        py::array_t<float, py::array::c_style | py::array::forcecast> env;
        if (!env_rgba.is_none()) {
            env = env_rgba.cast<py::array_t<float, py::array::c_style | py::array::forcecast>>();
            if (env.ndim() != 3 || env.shape(2) != 4) throw std::invalid_argument("env_rgba must be H x W x 4");
            d.env_height = (int)env.shape(0);
            d.env_width = (int)env.shape(1);
            d.env_rgba = env.data();
        }
        check(s_, pt_load_arrays(s_, &d));
        loaded();
    }

    int getWidth() const { return w_; }
    int getHeight() const { return h_; }
    SceneModel& getSceneModel() { return model_; }

    // used by SceneModel
    pt_session* handle() { return s_; }
    void edited() {  // render_session.cu:109-110: m_pathTracer->reset(); m_sppOptimizer.reset()
        finish();
        check(s_, pt_reset(s_));
        optimizer_.reset();
    }
    void finish() {
        if (in_flight_) {
            float ms = 0.f;
            check(s_, pt_wait(s_, &ms));
            in_flight_ = false;
            optimizer_.track(frame_spp_, ms);
            int spp = 0;
            check(s_, pt_get_spp(s_, &spp));
            model_.updateSpp(spp);
        }
    }
    void snapshot(int spp) {
        if (snapshot_.empty()) return;
        for (int t = 2; t <= (1 << 20); t <<= 1)
            if (spp >= t && spp - frame_spp_ < t) {
                check(s_, pt_save_exr(s_, snapshot_.c_str()));
                snapshots_++;
                break;
            }
    }
    int snapshots_ = 0;
    std::string snapshot_;
    int max_depth_ = 5;
    bool nee_ = true;
    int num_materials_ = 0;

private:
    void loaded() {
        pt_scene_counts c;
        check(s_, pt_scene_counts_get(s_, &c));
        max_depth_ = c.default_depth;
        nee_ = c.default_nee != 0;
        num_materials_ = c.num_materials;
        model_.setMaterialID(-1);
        model_.updateSpp(0);
        optimizer_.reset();
    }
    void require_init() const {
        if (!initialised_) throw std::runtime_error("RenderSession.init() has not been called");
    }
    pt_session* s_ = nullptr;
    int w_, h_;
    SceneModel model_;
    SppOptimizer optimizer_;
    bool initialised_ = false;
    bool in_flight_ = false;
    int frame_spp_ = 1;
};

SceneModel::Mat SceneModel::material(int id) const {
    Mat m{};
    if (id < 0 || id >= s_->num_materials_) return m;
    std::vector<int> types(s_->num_materials_);
    std::vector<float> albedo(3 * s_->num_materials_), emit(3 * s_->num_materials_), ior(s_->num_materials_),
        alpha(s_->num_materials_);
    pt_scene_export e{};
    e.material_types = types.data();
    e.material_albedo = albedo.data();
    e.material_emit = emit.data();
    e.material_ior = ior.data();
    e.material_alpha = alpha.data();
    check(s_->handle(), pt_export_scene(s_->handle(), &e));
    m.type = types[id];
    for (int k = 0; k < 3; k++) {
        m.albedo[k] = albedo[3 * id + k];
        m.emit[k] = emit[3 * id + k];
    }
    m.ior = ior[id];
    m.alpha = alpha[id];
    return m;
}

void SceneModel::apply(const Mat& m) {
    s_->finish();
    if (material_id_ >= 0)
        check(s_->handle(),
              pt_set_material(s_->handle(), material_id_, m.type, m.albedo, m.emit, m.ior, m.alpha));
    s_->edited();
}

void SceneModel::camera(float out[11]) const {
    pt_scene_export e{};
    e.camera = out;
    check(s_->handle(), pt_export_scene(s_->handle(), &e));
}

void SceneModel::set_camera(const float c[11]) {
    s_->finish();
    check(s_->handle(), pt_set_camera(s_->handle(), c, c + 3, c + 6, c[9], c[10] != 0.f ? 1 : 0));
    s_->edited();
}

// The renderer switch (render_session.cu:82-87, applied after the frame in flight,
// render_session.h:102-112): the CUDA path tracer or the normals G-buffer; no OptiX backend.
void SceneModel::setRendererType(RendererType t) {
    if (t == RendererType::Optix)
        throw std::runtime_error("no OptiX backend: the CUDA path tracer and the normals renderer are provided");
    s_->finish();
    check(s_->handle(), pt_set_renderer(s_->handle(), t == RendererType::Normals ? PT_RENDERER_NORMALS : PT_RENDERER_CUDA));
    renderer_ = t;
    s_->edited();
}

void SceneModel::setColor(float r, float g, float b) {
    Mat m = material(material_id_);
    m.albedo[0] = r; m.albedo[1] = g; m.albedo[2] = b;
    apply(m);
}
Vec3 SceneModel::getColor() const {
    if (material_id_ == -1) return Vec3{{0.f, 0.f, 0.f}};
    const Mat m = material(material_id_);
    return Vec3{{m.albedo[0], m.albedo[1], m.albedo[2]}};
}
void SceneModel::setEmit(float r, float g, float b) {
    Mat m = material(material_id_);
    m.emit[0] = r; m.emit[1] = g; m.emit[2] = b;
    apply(m);
}
Vec3 SceneModel::getEmit() const {
    if (material_id_ == -1) return Vec3{{0.f, 0.f, 0.f}};
    const Mat m = material(material_id_);
    return Vec3{{m.emit[0], m.emit[1], m.emit[2]}};
}
float SceneModel::getIOR() const { return material_id_ == -1 ? -1.f : material(material_id_).ior; }
void SceneModel::setIOR(float ior) {
    Mat m = material(material_id_);
    m.ior = ior;
    apply(m);
}
float SceneModel::getAlpha() const { return material_id_ == -1 ? -1.f : material(material_id_).alpha; }
void SceneModel::setAlpha(float alpha) {
    Mat m = material(material_id_);
    m.alpha = alpha;
    apply(m);
}
MaterialType SceneModel::getMaterialType() const {
    return material_id_ == -1 ? MaterialType::None : (MaterialType)material(material_id_).type;
}
void SceneModel::setMaterialType(MaterialType t) {
    if (t == MaterialType::None) throw std::runtime_error("MaterialType.None cannot be assigned");
    Mat m = material(material_id_);
    m.type = (int)t;  // a type change resets the other parameters to the type's defaults
    apply(m);
}
void SceneModel::setLightPosition(float p) {  // stored; the scene is unchanged (scene_model.cu:158-171)
    light_position_ = p;
    s_->edited();
}
Vec3 SceneModel::getCameraOrigin() const {
    float c[11];
    camera(c);
    return Vec3{{c[0], c[1], c[2]}};
}
void SceneModel::setCameraOrigin(float x, float y, float z) {
    float c[11];
    camera(c);
    c[0] = x; c[1] = y; c[2] = z;
    set_camera(c);
}
Vec3 SceneModel::getCameraTarget() const {
    float c[11];
    camera(c);
    return Vec3{{c[3], c[4], c[5]}};
}
void SceneModel::setCameraTarget(float x, float y, float z) {
    float c[11];
    camera(c);
    c[3] = x; c[4] = y; c[5] = z;
    set_camera(c);
}
Vec3 SceneModel::getCameraUp() const {
    float c[11];
    camera(c);
    return Vec3{{c[6], c[7], c[8]}};
}
void SceneModel::setCameraUp(float x, float y, float z) {
    float c[11];
    camera(c);
    c[6] = x; c[7] = y; c[8] = z;
    set_camera(c);
}
// scene_model.cu:268-289: the origin moves `ticks` along the normalised view direction
void SceneModel::zoomCamera(float ticks) {
    float c[11];
    camera(c);
    const float d[3] = {c[3] - c[0], c[4] - c[1], c[5] - c[2]};
    const float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (len > 0.f)
        for (int k = 0; k < 3; k++) c[k] += d[k] / len * ticks;
    set_camera(c);
}
int SceneModel::getMaxDepth() const { return s_->max_depth_; }
void SceneModel::setMaxDepth(int d) {
    s_->finish();
    check(s_->handle(), pt_set_max_depth(s_->handle(), d));
    s_->max_depth_ = d;
    s_->edited();
}
bool SceneModel::getNextEventEstimation() const { return s_->nee_; }
void SceneModel::setNextEventEstimation(bool on) {
    s_->finish();
    check(s_->handle(), pt_set_nee(s_->handle(), on ? 1 : 0));
    s_->nee_ = on;
    s_->edited();
}

}  // namespace

PYBIND11_MODULE(path_tracer, m) {
    m.doc() = "Path Tracer (B200 wavefront backend; headless)";

    py::class_<Vec3>(m, "Vec3")
        .def("x", &Vec3::x)
        .def("y", &Vec3::y)
        .def("z", &Vec3::z)
        .def("r", &Vec3::x)
        .def("g", &Vec3::y)
        .def("b", &Vec3::z)
        .def("__repr__", [](const Vec3& v) {
            return "Vec3(" + std::to_string(v.v[0]) + ", " + std::to_string(v.v[1]) + ", " +
                   std::to_string(v.v[2]) + ")";
        });

    py::class_<RenderState>(m, "RenderState")
        .def_readonly("isRendering", &RenderState::isRendering)
        .def_readonly("pbo", &RenderState::pbo);

    py::enum_<RendererType>(m, "RendererType")
        .value("CUDA", RendererType::CUDA)
        .value("Optix", RendererType::Optix)
        .value("Normals", RendererType::Normals)
        .export_values();

    py::enum_<MaterialType>(m, "MaterialType")
        .value("Lambertian", MaterialType::Lambertian)
        .value("Mirror", MaterialType::Mirror)
        .value("Glass", MaterialType::Glass)
        .value("Microfacet", MaterialType::Microfacet)
        .value("None", MaterialType::None)
        .value("Metal", MaterialType::Metal)
        .export_values();

    py::class_<MaterialIndex>(m, "MaterialIndex")
        .def_readonly("materialType", &MaterialIndex::materialType)
        .def_readonly("index", &MaterialIndex::index);

    py::class_<SceneModel>(m, "SceneModel")
        .def("getRendererType", &SceneModel::getRendererType)
        .def("setRendererType", &SceneModel::setRendererType)
        .def("setColor", &SceneModel::setColor)
        .def("getColor", &SceneModel::getColor)
        .def("setEmit", &SceneModel::setEmit)
        .def("getEmit", &SceneModel::getEmit)
        .def("getIOR", &SceneModel::getIOR)
        .def("setIOR", &SceneModel::setIOR)
        .def("getAlpha", &SceneModel::getAlpha)
        .def("setAlpha", &SceneModel::setAlpha)
        .def("getMaterialID", &SceneModel::getMaterialID)
        .def("getMaterialType", &SceneModel::getMaterialType)
        .def("setMaterialType", &SceneModel::setMaterialType)
        .def("setLightPosition", &SceneModel::setLightPosition)
        .def("getLightPosition", &SceneModel::getLightPosition)
        .def("getCameraOrigin", &SceneModel::getCameraOrigin)
        .def("setCameraOrigin", &SceneModel::setCameraOrigin)
        .def("getCameraTarget", &SceneModel::getCameraTarget)
        .def("setCameraTarget", &SceneModel::setCameraTarget)
        .def("getCameraUp", &SceneModel::getCameraUp)
        .def("setCameraUp", &SceneModel::setCameraUp)
        .def("getMaxDepth", &SceneModel::getMaxDepth)
        .def("setMaxDepth", &SceneModel::setMaxDepth)
        .def("getNextEventEstimation", &SceneModel::getNextEventEstimation)
        .def("setNextEventEstimation", &SceneModel::setNextEventEstimation)
        .def("zoomCamera", &SceneModel::zoomCamera)
        .def("getSpp", &SceneModel::getSpp);

    py::class_<Session>(m, "RenderSession")
        .def(py::init<int, int, int, uint64_t>(), py::arg("width"), py::arg("height"), py::arg("config") = 0,
             py::arg("seed") = 0x5EEDULL)
        .def("init", &Session::init, "Initialize CUDA resources (no GL buffers: headless)")
        .def("renderAsync", &Session::renderAsync, "Render and update buffer")
        .def("pollRender", &Session::pollRender, "Poll the render state")
        .def("hitTest", &Session::hitTest, "Run a material hit test")
        .def("getWidth", &Session::getWidth)
        .def("getHeight", &Session::getHeight)
        .def("getSceneModel", &Session::getSceneModel, py::return_value_policy::reference_internal)
        .def("getRadianceBuffer", &Session::getRadianceBuffer, "Progressive radiance, H x W x 3 FP32")
        .def("readback", &Session::getRadianceBuffer, "Progressive radiance, H x W x 3 FP32 (row 0 = bottom)")
        .def("readback_rgba8", &Session::readbackRGBA8, "Display bytes, H x W x 4 (sRGB)")
        .def("load_scene", &Session::loadScene, py::arg("config_id"), py::arg("seed") = 0x5EEDULL,
             "Load generated configuration 0-3")
        .def("setSnapshotPath", &Session::setSnapshotPath, py::arg("path"),
             "Write the radiance buffer as EXR at every power-of-two spp (render_session.h:87-101); '' = off")
        .def("getSnapshotPath", &Session::getSnapshotPath)
        .def_readonly("snapshots", &Session::snapshots_)
        .def("load_reference_scene", &Session::loadReferenceScene, py::arg("index"), py::arg("scenes_dir"),
             "Load the reference's built-in scene 0-3 (OBJ/MTL, PLY and EXR files of its scenes/ directory)")
        .def("load_scene_arrays", &Session::loadSceneArrays, py::arg("tri_vertices"), py::arg("tri_normals"),
             py::arg("tri_materials"), py::arg("spheres"), py::arg("sphere_materials"), py::arg("material_types"),
             py::arg("material_albedo"), py::arg("material_emit"), py::arg("material_ior"),
             py::arg("material_alpha"), py::arg("env_rgba") = py::none(),
             "Load a scene from arrays (triangles 9 floats, spheres 4 floats, per-material parameters)");
}
