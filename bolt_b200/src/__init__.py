"""Physics plug-ins recognised by the native solver path."""
