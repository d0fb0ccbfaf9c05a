"""Gradients of the detected count and mean arrival time (the gradient replay
kernel, g4b_gradients) against central finite differences with common random
numbers, through a torch.autograd.Function.

Parameters: the crystal's refractive index n, its absorption length L, the
wrapper reflectivity R and the scintillation decay time tau, on 2,000 events
of 5 MeV electrons (FP32 forward, FP32 replay with FP64 accumulation). The
finite differences use relative steps of 1e-3 and the same gensteps and seed;
the tolerance is the north_star's 2 %.
"""
import numpy as np
import pytest
import torch

from g4go_b200 import PhotonTransportBatch, PhotonTransportConfig, TransportHost, scenes

pytestmark = pytest.mark.gpu

PARAMETERS = ("rindex", "abs_length_mm", "reflectivity", "decay_time_ns")
SEED = 424242


def with_decay(batch, tau):
    emissions = batch.emissions.copy()
    scint = emissions["type"] == 2
    emissions["decay_time_ns"][scint] = np.float32(tau)
    return PhotonTransportBatch(emissions, batch.event_ids, batch.emission_event_indices)


def evaluate(theta, base, gradients=False):
    n, length, reflectivity, tau = (float(x) for x in theta)
    scene = scenes.crystal_sipm_scene(scenes.DetectorParameters(
        crystal_rindex=n, crystal_abs_length_mm=length, wrapper_reflectivity=reflectivity))
    batch = with_decay(base, tau)
    with TransportHost(PhotonTransportConfig(seed=SEED, precision="fp32")) as host:
        host.enqueue_emissions(scene, batch)
        out = host.complete_oldest_batch()
        grads = host.gradients(scenes.MAT_CRYSTAL, scenes.MAT_CRYSTAL, scenes.SURF_WRAPPER) if gradients else None
    detected = float(out.statistics["detected_count"])
    mean_time = float(np.mean(out.detections["time_ns"].astype(np.float64)))
    return detected, mean_time, grads


class DetectorResponse(torch.autograd.Function):
    """theta = (n, L, R, tau) -> (detected count, mean arrival time) on the GPU engine."""

    @staticmethod
    def forward(ctx, theta, base):
        detected, mean_time, grads = evaluate(theta.detach().cpu().numpy(), base, gradients=True)
        assert grads["replay_mismatches"] == 0
        jacobian = torch.tensor([[grads["d_detected"][p] for p in PARAMETERS],
                                 [grads["d_mean_time_ns"][p] for p in PARAMETERS]], dtype=torch.float64)
        ctx.save_for_backward(jacobian)
        return torch.tensor([detected, grads["mean_time_ns"]], dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_output):
        (jacobian,) = ctx.saved_tensors
        return grad_output @ jacobian, None


@pytest.fixture(scope="module")
def base_batch():
    return scenes.workload("gradients", seed=5)


@pytest.mark.parametrize("theta0", [(1.82, 400.0, 0.95, 40.0), (1.74, 150.0, 0.85, 25.0)])
def test_gradients_match_central_differences(base_batch, theta0):
    theta = torch.tensor(theta0, dtype=torch.float64, requires_grad=True)
    response = DetectorResponse.apply(theta, base_batch)
    (grad_detected,) = torch.autograd.grad(response[0], theta, retain_graph=True)
    (grad_time,) = torch.autograd.grad(response[1], theta)
    step = 1e-3
    report = []
    for j, name in enumerate(PARAMETERS):
        h = step * theta0[j]
        plus = list(theta0)
        minus = list(theta0)
        plus[j] += h
        minus[j] -= h
        n_plus, t_plus, _ = evaluate(plus, base_batch)
        n_minus, t_minus, _ = evaluate(minus, base_batch)
        fd_detected = (n_plus - n_minus) / (2 * h)
        fd_time = (t_plus - t_minus) / (2 * h)
        report.append((name, grad_detected[j].item(), fd_detected, grad_time[j].item(), fd_time))
    print("\nparameter  dN/dtheta (replay, FD)  dT/dtheta (replay, FD)")
    for name, gd, fd, gt, ft in report:
        print(f"{name:14s} {gd:14.6g} {fd:14.6g}   {gt:12.6g} {ft:12.6g}")
    for name, gd, fd, gt, ft in report:
        if name == "decay_time_ns":
            assert gd == 0.0 and fd == 0.0  # the decay time moves arrival times only
        else:
            assert abs(gd - fd) <= 0.02 * abs(fd), (name, "detected", gd, fd)
        assert abs(gt - ft) <= 0.02 * abs(ft) + 1e-9, (name, "mean time", gt, ft)
