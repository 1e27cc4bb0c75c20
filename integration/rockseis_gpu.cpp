// Definitions of the specialisations declared in rockseis_gpu.h: the bodies of
// ModellingAcoustic2D<float>::run, ModellingElastic2D<float>::run and
// FwiAcoustic2D<float>::run_optimal rewritten as calls to the C ABI of
// librsgpu (include/rsgpu.h).  The reference objects are passed as they are:
// padded staggered parameters from the Model getters, SMAP/GMAP maps and shifts
// from the Geometry2D, wavelets and traces in the Data2D arrays (traces are
// accumulated like recordData).  RSGPU_F32_EXACT makes the results identical
// bit for bit to the CPU bodies they replace.
//
// Not carried over: wavefield snapshots (Modelling::setSnapP/Vx/Vz) and FWI data
// weights (Fwi*::setDataweight); a run that asks for them stops with rs_error.
#include <cstdlib>
#include <vector>

#include "rockseis_gpu.h"
#include "rsgpu.h"

namespace rockseis {
namespace {

// The C-PML tables of a run (the Pml object WavesAcoustic2D/WavesElastic2D build
// with Smax = SMAX), in rsgpu_config.pml order.
std::vector<float> pml_tables(int lpml, float dt)
{
    Pml<float> p(lpml, dt);
    p.setSmax(SMAX);
    p.computeABC();
    const float *tab[12] = {p.A_ltf, p.B_ltf, p.C_ltf, p.A_ltf_stag, p.B_ltf_stag, p.C_ltf_stag,
                            p.A_rbb, p.B_rbb, p.C_rbb, p.A_rbb_stag, p.B_rbb_stag, p.C_rbb_stag};
    std::vector<float> out((size_t)12 * lpml);
    for (int k = 0; k < 12; k++)
        for (int i = 0; i < lpml; i++) out[(size_t)k * lpml + i] = tab[k][i];
    return out;
}

rsgpu_config base_config(int physics, int lpml, int order, int fs, int nt, double dx, double dz, double dt,
                         const float *pml)
{
    rsgpu_config c = {};
    c.physics = physics;
    c.precision = RSGPU_F32_EXACT;
    c.lpml = lpml;
    c.order = order;
    c.fs = fs;
    c.nt = nt;
    c.dx = dx;
    c.dy = 1.0;
    c.dz = dz;
    c.dt = dt;
    c.pml = pml;
    c.tile = -1;
    return c;
}

// source part of a shot (SMAP)
void set_source(rsgpu_shot &s, const std::shared_ptr<Data2D<float>> &src)
{
    s.nsrc = (int)src->getNtrace();
    s.smap = &src->getGeom()->getSmap()[0].x;
    s.sshift = &src->getGeom()->getSshift()[0].x;
    s.wavelet = src->getData();
    s.src_field = (int)src->getField();
}

// receiver part of a shot (GMAP), traces accumulated into rec's data
void set_receivers(rsgpu_shot &s, const std::shared_ptr<Data2D<float>> &rec, int field)
{
    s.nrec = (int)rec->getNtrace();
    s.gmap = &rec->getGeom()->getGmap()[0].x;
    s.gshift = &rec->getGeom()->getGshift()[0].x;
    s.rec_field = field;
    s.rec_out = rec->getData();
}

void check(rsgpu_status st, const char *who)
{
    if (st != RSGPU_OK) rs_error(who, rsgpu_last_error());
}

}  // namespace

template <>
int ModellingAcoustic2D<float>::run()
{
    if (!this->checkStability())
        rs_error("ModellingAcoustic2D::run: Wavelet sampling interval (dt) does not match the stability criteria.");
    if (this->snapPset || this->snapVxset || this->snapVzset)
        rs_error("ModellingAcoustic2D::run: snapshots are not produced by the GPU path.");
    this->createLog(this->getLogfile());
    this->writeLog("Running 2D Acoustic modelling.");
    const std::vector<float> pml = pml_tables(model->getLpml(), source->getDt());
    rsgpu_config cfg = base_config(RSGPU_ACOUSTIC2D, model->getLpml(), this->getOrder(), model->getFs(),
                                   source->getNt(), model->getDx(), model->getDz(), source->getDt(), pml.data());
    rsgpu_shot proto = {};
    proto.nx = model->getNx();
    proto.ny = 1;
    proto.nz = model->getNz();
    proto.model[0] = model->getRx();
    proto.model[1] = model->getRz();
    proto.model[2] = model->getL();
    set_source(proto, source);
    // one batch entry per receiver set (P, Vx, Vz), all recorded from the same run
    std::vector<rsgpu_shot> shots;
    const std::shared_ptr<Data2D<float>> sets[3] = {recP, recVx, recVz};
    const bool on[3] = {recPset, recVxset, recVzset};
    for (int k = 0; k < 3; k++) {
        if (!on[k]) continue;
        rsgpu_shot s = proto;
        set_receivers(s, sets[k], (int)sets[k]->getField());
        shots.push_back(s);
    }
    if (shots.empty()) shots.push_back(proto);
    check(rsgpu_modelling(&cfg, (int)shots.size(), shots.data()), "ModellingAcoustic2D::run: ");
    this->writeLog("Modelling is complete.");
    return MOD_OK;
}

template <>
int ModellingElastic2D<float>::run()
{
    if (!this->checkStability())
        rs_error("ModellingElastic2D::run: Wavelet sampling interval (dt) does not match the stability criteria.");
    if (this->snapPset || this->snapVxset || this->snapVzset)
        rs_error("ModellingElastic2D::run: snapshots are not produced by the GPU path.");
    this->createLog(this->getLogfile());
    this->writeLog("Running 2D Elastic modelling.");
    const std::vector<float> pml = pml_tables(model->getLpml(), source->getDt());
    rsgpu_config cfg = base_config(RSGPU_ELASTIC2D, model->getLpml(), this->getOrder(), model->getFs(),
                                   source->getNt(), model->getDx(), model->getDz(), source->getDt(), pml.data());
    rsgpu_shot proto = {};
    proto.nx = model->getNx();
    proto.ny = 1;
    proto.nz = model->getNz();
    proto.model[0] = model->getRx();
    proto.model[1] = model->getRz();
    proto.model[2] = model->getL();
    proto.model[3] = model->getL2M();
    proto.model[4] = model->getM();
    set_source(proto, source);
    std::vector<rsgpu_shot> shots;
    std::vector<std::vector<float>> factors;
    factors.reserve(3);
    const std::shared_ptr<Data2D<float>> sets[3] = {recP, recVx, recVz};
    const bool on[3] = {recPset, recVxset, recVzset};
    for (int k = 0; k < 3; k++) {
        if (!on[k]) continue;
        rsgpu_shot s = proto;
        set_receivers(s, sets[k], (int)sets[k]->getField());
        if (k == 0 && recP->getReciprocity()) {
            // R*Vp*Vp - R*Vs*Vs at each receiver cell (WavesElastic2D::recordData)
            const int nx = model->getNx();
            const float *R = model->getR(), *Vp = model->getVp(), *Vs = model->getVs();
            const Point2D<int> *map = recP->getGeom()->getGmap();
            std::vector<float> f((size_t)s.nrec, 1.0f);
            for (int t = 0; t < s.nrec; t++)
                if (map[t].x >= 0 && map[t].y >= 0) {
                    const size_t c = (size_t)map[t].y * nx + map[t].x;
                    f[t] = R[c] * Vp[c] * Vp[c] - R[c] * Vs[c] * Vs[c];
                }
            factors.push_back(f);
            s.rec_factor = factors.back().data();
        }
        shots.push_back(s);
    }
    if (shots.empty()) shots.push_back(proto);
    check(rsgpu_modelling(&cfg, (int)shots.size(), shots.data()), "ModellingElastic2D::run: ");
    this->writeLog("Modelling is complete.");
    return MOD_OK;
}

template <>
int FwiAcoustic2D<float>::run_optimal()
{
    if (!vpgradset && !rhogradset) {
        rs_warning("FwiAcoustic2D::run: No image set");
        return FWI_ERR;
    }
    if (dataweightset) rs_error("FwiAcoustic2D::run_optimal: data weights are not applied by the GPU path.");
    this->createLog(this->getLogfile());
    this->writeLog("Running 2D Acoustic full-waveform inversion gradient with optimal checkpointing.");
    if (vpgradset) vpgrad->allocateImage();
    if (rhogradset) rhograd->allocateImage();
    if (srcilumset) srcilum->allocateImage();
    const std::vector<float> pml = pml_tables(model->getLpml(), source->getDt());
    rsgpu_config cfg = base_config(RSGPU_ACOUSTIC2D, model->getLpml(), this->getOrder(), model->getFs(),
                                   source->getNt(), model->getDx(), model->getDz(), source->getDt(), pml.data());
    rsgpu_adjoint_opts o = {};
    o.ncheck = this->getNcheck();
    o.ckpt_precision = RSGPU_CKPT_NATIVE;
    o.accum = RSGPU_ACCUM_REFERENCE;
    o.misfit = (int)this->getMisfit_type();
    o.nhx = o.nhz = o.nhy = 1;
    rsgpu_adjoint_shot a = {};
    a.shot.nx = model->getNx();
    a.shot.ny = 1;
    a.shot.nz = model->getNz();
    a.shot.model[0] = model->getRx();
    a.shot.model[1] = model->getRz();
    a.shot.model[2] = model->getL();
    set_source(a.shot, source);
    set_receivers(a.shot, dataP, RSGPU_PRESSURE);
    a.shot.rec_out = datamodPset ? datamodP->getData() : nullptr;
    a.vp = model->getVp();
    a.rho = model->getR();
    a.data = dataP->getData();
    a.vpgrad = vpgradset ? vpgrad->getImagedata() : nullptr;
    a.rhograd = rhogradset ? rhograd->getImagedata() : nullptr;
    a.wavgrad = wavgradset ? wavgrad->getData() : nullptr;
    a.datares = dataresPset ? dataresP->getData() : nullptr;
    a.srcilum = srcilumset ? srcilum->getImagedata() : nullptr;
    double mis = 0.0;
    a.misfit = &mis;
    check(rsgpu_fwi_gradient(&cfg, &o, 1, &a), "FwiAcoustic2D::run_optimal: ");
    this->setMisfit((float)mis);
    this->writeLog("\nGradient computation completed.");
    return FWI_OK;
}

}  // namespace rockseis
