"""The drop-in layer: reference OPS applications, unmodified, on OPS-B200
(see ops_dropin.h)."""
