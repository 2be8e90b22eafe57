"""Device selection helpers with the behaviour of ``torchcor/device.py:3-33``."""
import torch


def set_device(name=None, verbose=True):
    """Make ``name`` (default: the first CUDA device) the current device."""
    device = torch.device("cuda" if torch.cuda.is_available() else "cpu") if name is None else torch.device(name)
    if torch.cuda.is_available():
        torch.cuda.set_device(device)
        if verbose:
            i = torch.cuda.current_device()
            props = torch.cuda.get_device_properties(i)
            print(f"GPU: {torch.cuda.get_device_name(i)}", flush=True)
            print(f"Total Memory: {props.total_memory / (1024 ** 3):.2f} GB", flush=True)
    elif verbose:
        print("No GPU available. Using CPU instead.", flush=True)


def get_device():
    """The current CUDA device, or ``cpu`` when no GPU is present."""
    if torch.cuda.is_available():
        return torch.device(f"cuda:{torch.cuda.current_device()}")
    return torch.device("cpu")
